"""Benchmark of the index step (k-mers/s), the configuration the headline
metric is quoted on: a 100 Mbp reference (40 genomes of 2.5 Mbp, each derived
from one of 4 random founders by 2% substitutions + 0.1% indels), k = 31,
both strands; 10 M reads with log-normal lengths (median 150, clipped to
31..1000), 0.5% substitutions, 0.1% N.  All data is seeded synthetic data
generated at start-up by the project's tools.

One step = one index-step pass (SeqToBits + positions + SBWT search + -1/-2
mapping) over the whole read batch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` = k-mers/s with inputs resident in HBM
(device-pointer call); `e2e` = the same through the host-pointer C-ABI call
from pinned host memory (H2D + compute + D2H inside the timed region).
Multi-GPU: one process per GPU (torchrun), each rank searches its own read
batch against its own index replica (no collective on the data path; weak
scaling).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "sbwt-search_b200"))

METRIC = "k-mers/s index search (reads -> SBWT index per k-mer)"
UNIT = "k-mers/s"

CFG = dict(n_genomes=40, genome_len=2_500_000, n_founders=4, sub=0.02, indel=0.001,
           k=31, n_reads=10_000_000, len_median=150, len_sigma=0.5, len_min=31,
           len_max=1000, read_sub=0.005, n_rate=0.001)


# pseudoalignment workload: 2000 genomes of 100 kbp from 8 random founders at
# 1-5 % divergence, k = 31, both strands; 5 M reads of 150 bp from random
# genomes with 0.5 % substitutions; tau = 0.7, not-found / invalid excluded.
CFG3 = dict(n_genomes=2000, genome_len=100_000, n_founders=8, sub_lo=0.01, sub_hi=0.05,
            k=31, n_reads=5_000_000, read_len=150, read_sub=0.005, tau=0.7)
# batched mixed workload against the index above: 256 files, read counts
# log-uniform in [50, 1e5] (the [1e3, 2e6] of the full-size workload scaled
# by 1/20 in read count so that it fits the default run), 10 % of the files
# with 1-10 kbp reads, the rest 100 bp, 5 % substitutions.
CFG4 = dict(n_files=256, reads_lo=50, reads_hi=100_000, long_frac=0.1, short_len=100,
            long_lo=1000, long_hi=10_000, sub=0.05)


def bench_batched(args, idx, S, torch, dev, scratch):
    """Batched (one call over all files = one persistent launch fed by the
    device work queue, after the autotuner) vs plain (one call per file, the
    reference's per-file launch pattern), device-resident, bit-exact."""
    import sbwt_tools as T
    rng = np.random.default_rng(7)
    g = T.gen_genomes(20240601, CFG["n_genomes"], CFG["genome_len"], CFG["n_founders"],
                      CFG["sub"], CFG["sub"], CFG["indel"])
    files = []
    for f in range(CFG4["n_files"]):
        n = int(np.exp(rng.uniform(np.log(CFG4["reads_lo"]), np.log(CFG4["reads_hi"]))))
        if rng.random() < CFG4["long_frac"]:
            ch, en = T.gen_reads(9000 + f, g, n, 1.0, 3000, 0.6, CFG4["long_lo"],
                                 CFG4["long_hi"], CFG4["sub"], 0.0)
        else:
            ch, en = T.gen_reads(9000 + f, g, n, 1.0, CFG4["short_len"], 0.0,
                                 CFG4["short_len"], CFG4["short_len"], CFG4["sub"], 0.0)
        files.append((ch, en))
    chars = np.concatenate([f[0] for f in files])
    base = np.cumsum([0] + [len(f[0]) for f in files])[:-1]
    ends = np.concatenate([f[1] + b for f, b in zip(files, base)]).astype(np.uint64)
    n_k = idx.count_kmers(ends)
    d_chars = torch.from_numpy(chars).to(f"cuda:{dev}")
    d_ends = torch.from_numpy(ends.view(np.int64)).to(f"cuda:{dev}")
    d_out = torch.empty(n_k, dtype=torch.int64, device=f"cuda:{dev}")
    # plain: one call per file (each call synchronises, as the reference's
    # per-batch copy-kernel-copy does)
    fk = [idx.count_kmers(f[1]) for f in files]
    koff = np.cumsum([0] + fk)
    d_files = [(torch.from_numpy(f[0]).to(f"cuda:{dev}"),
                torch.from_numpy(f[1].view(np.int64)).to(f"cuda:{dev}")) for f in files]
    d_plain = torch.empty(n_k, dtype=torch.int64, device=f"cuda:{dev}")
    S.set_launch_config()

    def plain():
        for i, (dc, de) in enumerate(d_files):
            if fk[i]:
                idx.search_reads(dc, de, out=d_plain[int(koff[i]):int(koff[i + 1])])

    plain()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain()
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    tune = S.autotune(idx, d_chars, d_ends, sample_chars=64 << 20, use_cache=False)
    idx.search_reads(d_chars, d_ends, out=d_out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        idx.search_reads(d_chars, d_ends, out=d_out)
    e1.record()
    torch.cuda.synchronize()
    t_batch = e0.elapsed_time(e1) / 3 / 1e3
    exact = bool(torch.equal(d_out, d_plain))
    S.set_launch_config()
    S.set_table_kernel(args.kernel)
    S.set_block_threads(256)
    return {"workload": "256 files vs the 100 Mbp index, reads/file log-uniform [50, 1e5] "
                        "(full-size range [1e3, 2e6] scaled 1/20), 10% files of 1-10 kbp "
                        "reads, 5% substitutions", "files": len(files),
            "reads": int(len(ends)), "kmers": int(n_k),
            "batched_kmers_per_s": n_k / t_batch, "plain_kmers_per_s": n_k / t_plain,
            "speedup": t_plain / t_batch, "bit_exact": exact, "autotune": tune}


# batched mixed workload at its full size: 256 files, reads/file log-uniform in
# [1e3, 2e6], 10 % of the files with 1-10 kbp reads, the rest 100 bp, 5 %
# substitutions (about 4.5e10 chars in all).
CFG4_FULL = dict(n_files=256, reads_lo=1_000, reads_hi=2_000_000, long_frac=0.1,
                 short_len=100, long_lo=1000, long_hi=10_000, sub=0.05,
                 short_pool=2_000_000, long_pool=100_000, wave_chars=3_000_000_000)


def _wave_checksum(torch, out, n):
    """Position-weighted wrapping sum of the first n results (chunked)."""
    total = torch.zeros((), dtype=torch.int64, device=out.device)
    step = 1 << 27
    for lo in range(0, n, step):
        hi = min(n, lo + step)
        w = torch.arange(2 * lo + 1, 2 * hi + 1, 2, dtype=torch.int64, device=out.device)
        total += (out[lo:hi] * w).sum()
    return int(total.item())


def bench_batched_full(args, idx, S, torch, dev):
    """The batched workload at its stated size, streamed in waves of files
    that fit the device: the files' reads are cyclic runs of two seeded read
    pools kept on the device (2 M short reads, 100 k long reads), so a wave
    is assembled by device copies.  Per wave: plain = one sbwt_search_reads
    call per file (each synchronous, the library defaults); batched = one
    call over the whole wave (one persistent launch), with the library
    defaults and with the autotuner's choice.  Bit-exact: equal
    position-weighted checksums of all results and equal first 1 M results
    of every wave."""
    import sbwt_tools as T
    c = CFG4_FULL
    rng = np.random.default_rng(17)
    g = T.gen_genomes(20240601, CFG["n_genomes"], CFG["genome_len"], CFG["n_founders"],
                      CFG["sub"], CFG["sub"], CFG["indel"])
    pools = {}
    for kind, n, med, sig, lo, hi in (("short", c["short_pool"], c["short_len"], 0.0,
                                       c["short_len"], c["short_len"]),
                                      ("long", c["long_pool"], 3000, 0.6, c["long_lo"],
                                       c["long_hi"])):
        ch, en = T.gen_reads(4242 + len(pools), g, n, 1.0, med, sig, lo, hi, c["sub"], 0.0)
        lens = np.diff(np.concatenate([[0], en.astype(np.int64)]))
        pools[kind] = (torch.from_numpy(ch).to(f"cuda:{dev}"), lens,
                       np.concatenate([[0], np.cumsum(lens)]))
    files = []
    for f in range(c["n_files"]):
        n = int(np.exp(rng.uniform(np.log(c["reads_lo"]), np.log(c["reads_hi"]))))
        kind = "long" if rng.random() < c["long_frac"] else "short"
        files.append((kind, int(rng.integers(0, len(pools[kind][1]))), n))

    def file_arrays(kind, start, n):
        d_ch, lens, cum = pools[kind]
        P = len(lens)
        segs, lsegs, left, s0 = [], [], n, start
        while left:
            take = min(left, P - s0)
            segs.append(d_ch[int(cum[s0]):int(cum[s0 + take])])
            lsegs.append(lens[s0:s0 + take])
            left -= take
            s0 = 0
        return segs, np.concatenate(lsegs)

    def file_chars(f):
        kind, start, n = files[f]
        lens = pools[kind][1]
        P = len(lens)
        full, rem = divmod(n, P)
        cum = pools[kind][2]
        tot = full * int(cum[P]) + (int(cum[min(start + rem, P)] - cum[start]) +
                                    (int(cum[start + rem - P]) if start + rem > P else 0))
        return tot

    # waves of consecutive files up to wave_chars (a larger file is a wave)
    waves, cur, cur_c = [], [], 0
    for f in range(len(files)):
        fc = file_chars(f)
        if cur and cur_c + fc > c["wave_chars"]:
            waves.append(cur)
            cur, cur_c = [], 0
        cur.append(f)
        cur_c += fc
    waves.append(cur)
    stream = torch.cuda.current_stream(dev)
    tot = {"plain": 0.0, "batched": 0.0, "batched_tuned": 0.0, "plain_tuned": 0.0}
    n_kmers = n_chars = n_reads = 0
    exact = True
    tune = None
    for wi, wave in enumerate(waves):
        segs, lens, fk, fr = [], [], [], []
        for f in wave:
            s_, l_ = file_arrays(*files[f])
            segs += s_
            lens.append(l_)
            fr.append(len(l_))
        d_chars = torch.cat(segs)
        lens = np.concatenate(lens)
        ends = np.cumsum(lens).astype(np.uint64)
        d_ends = torch.from_numpy(ends.view(np.int64)).to(f"cuda:{dev}")
        n_k = idx.count_kmers(ends)
        # per file: its chars, its ends (file-relative), its k-mer slots
        rb = np.concatenate([[0], np.cumsum(fr)])
        per_file = []
        for i in range(len(wave)):
            c0 = int(ends[rb[i] - 1]) if rb[i] else 0
            c1 = int(ends[rb[i + 1] - 1])
            e = torch.from_numpy((ends[rb[i]:rb[i + 1]] - c0).view(np.int64)).to(f"cuda:{dev}")
            per_file.append((d_chars[c0:c1], e, idx.count_kmers(ends[rb[i]:rb[i + 1]] - c0)))
        koff = np.concatenate([[0], np.cumsum([x[2] for x in per_file])])
        d_out = torch.empty(n_k, dtype=torch.int64, device=f"cuda:{dev}")

        def plain():
            for i, (dc, de, k_) in enumerate(per_file):
                if k_:
                    idx.search_reads(dc, de, out=d_out[int(koff[i]):int(koff[i + 1])])
            torch.cuda.synchronize()

        def batched():
            idx.search_reads(d_chars, d_ends, out=d_out)
            torch.cuda.synchronize()

        def timed(fn):
            fn()  # warm (per-call workspaces grown)
            t0 = time.perf_counter()
            fn()
            return time.perf_counter() - t0

        S.set_launch_config()
        tot["plain"] += timed(plain)
        ref_ck = _wave_checksum(torch, d_out, n_k)
        ref_head = d_out[:1 << 20].clone()
        tot["batched"] += timed(batched)
        exact &= _wave_checksum(torch, d_out, n_k) == ref_ck
        exact &= bool(torch.equal(d_out[:1 << 20], ref_head))
        if tune is None:  # the autotuner on the first wave, kept for the rest
            tune = S.autotune(idx, d_chars, d_ends, sample_chars=256 << 20, use_cache=False)
        else:
            S.set_launch_config(presearch_letters=tune["presearch"],
                                blocks_per_sm=tune["blocks_per_sm"], tile=tune["tile"])
            S.set_table_kernel(tune["table_kernel"])
            S.set_block_threads(tune["block_threads"])
        tot["batched_tuned"] += timed(batched)
        exact &= _wave_checksum(torch, d_out, n_k) == ref_ck
        tot["plain_tuned"] += timed(plain)
        exact &= _wave_checksum(torch, d_out, n_k) == ref_ck
        S.set_launch_config()
        S.set_table_kernel(args.kernel)
        S.set_block_threads(256)
        n_kmers += n_k
        n_chars += int(ends[-1])
        n_reads += len(ends)
        del d_out, d_chars, d_ends, per_file, segs
        torch.cuda.empty_cache()
    del pools
    torch.cuda.empty_cache()
    return {"workload": "256 files vs the 100 Mbp index at the stated size: reads/file "
                        "log-uniform [1e3, 2e6], 10% files of 1-10 kbp reads (log-normal, "
                        "median 3 kbp), the rest 100 bp, 5% substitutions; reads are cyclic "
                        "runs of two seeded pools (2 M short, 100 k long reads) on the "
                        "device; processed in waves of <= 3e9 chars (a larger wave, or a "
                        "larger file, runs on the 64-bit kernel: > 2^32 k-mer slots)",
            "files": len(files), "waves": len(waves), "reads": int(n_reads),
            "chars": int(n_chars), "kmers": int(n_kmers),
            "plain_kmers_per_s": n_kmers / tot["plain"],
            "batched_kmers_per_s": n_kmers / tot["batched"],
            "plain_autotuned_kmers_per_s": n_kmers / tot["plain_tuned"],
            "batched_autotuned_kmers_per_s": n_kmers / tot["batched_tuned"],
            "speedup_same_launch_config": tot["plain"] / tot["batched"],
            "speedup_autotuned": tot["plain_tuned"] / tot["batched_tuned"],
            "speedup": tot["plain"] / tot["batched_tuned"],
            "bit_exact": bool(exact), "autotune": tune,
            "timing": "wall time around device-resident calls, each wave synchronised; "
                      "chars assembled on the device outside the timed calls"}


def colors_cli_file_to_file(sp, cp, chars, ends, tau, tmpdir):
    """The reference's two command lines on all reads of the colors workload,
    file to file: `sbwt_search index` (FASTQ -> ascii index results) then
    `sbwt_search colors` (index results -> ascii color ids), each timed with
    its process start and index load (an empty query measures those)."""
    cli = str(REPO / "sbwt-search_b200" / "_build" / "sbwt_search")
    fq = os.path.join(tmpdir, "colors_reads.fq")
    with open(fq, "wb") as f:
        for lo in range(0, len(ends), 1_000_000):
            hi = min(len(ends), lo + 1_000_000)
            base = int(ends[lo - 1]) if lo else 0
            f.write(fastq_text(chars[base:int(ends[hi - 1])], ends[lo:hi] - base).tobytes())
    idx_out, col_out = os.path.join(tmpdir, "colors_idx"), os.path.join(tmpdir, "colors_ids")
    empty = os.path.join(tmpdir, "colors_empty.fq")
    open(empty, "wb").close()

    def timed(argv):
        t0 = time.perf_counter()
        r = subprocess.run([cli, *argv], capture_output=True)
        return time.perf_counter() - t0, r.returncode

    t_idx_load, rc0 = timed(["index", "-i", sp, "-q", empty, "-o", idx_out + "_e"])
    t_idx, rc1 = timed(["index", "-i", sp, "-q", fq, "-o", idx_out])
    idx_bytes = os.path.getsize(idx_out + ".txt") if rc1 == 0 else 0
    os.remove(fq)
    # the colors step's empty query: an index results file of no reads
    with open(idx_out + "_e.txt", "rb") as f:
        hdr = f.read()
    with open(os.path.join(tmpdir, "colors_empty_idx.txt"), "wb") as f:
        f.write(hdr)
    t_col_load, rc2 = timed(["colors", "-k", cp, "-q", os.path.join(tmpdir, "colors_empty_idx.txt"),
                             "-o", col_out + "_e", "-t", str(tau)])
    t_col, rc3 = timed(["colors", "-k", cp, "-q", idx_out + ".txt", "-o", col_out, "-t",
                        str(tau)])
    col_bytes = os.path.getsize(col_out + ".txt") if rc3 == 0 else 0
    for x in (idx_out + ".txt", col_out + ".txt"):
        try:
            os.remove(x)
        except OSError:
            pass
    n = len(ends)
    return {"commands": "sbwt_search index -i <colors .sbwt> -q <reads FASTQ> -o <idx>; "
                        "sbwt_search colors -k <.tcolors> -q <idx>.txt -o <ids> -t 0.7 "
                        "(ascii in and out)",
            "reads": int(n), "rc": [rc0, rc1, rc2, rc3],
            "index_results_bytes": int(idx_bytes), "color_ids_bytes": int(col_bytes),
            "index_step_s": t_idx, "index_step_load_s": t_idx_load,
            "colors_step_s": t_col, "colors_step_load_s": t_col_load,
            "reads_per_s_both_steps_file_to_file":
                n / max(t_idx - t_idx_load + t_col - t_col_load, 1e-9),
            "reads_per_s_both_steps_incl_loads": n / max(t_idx + t_col, 1e-9)}


def bench_colors_and_serving(args, S, torch, dev, tmpdir, rank, resident_index=None):
    """Pseudoalignment reads/s (colors step, device-resident), the fused
    reads -> colors pipeline (host in, host out), the CPU oracle on a sample,
    and the serving loop's p50 / p99 latency at Poisson offered loads."""
    import threading
    import sbwt_tools as T
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    c = CFG3
    t0 = time.time()
    g = T.gen_genomes(33, c["n_genomes"], c["genome_len"], c["n_founders"], c["sub_lo"],
                      c["sub_hi"], 0.0)
    sp, cp = os.path.join(tmpdir, "cfg3.sbwt"), os.path.join(tmpdir, "cfg3.tcolors")
    t_b = time.time()
    nodes = T.build_colored(g, c["k"], sp, cp)
    t_host_build = time.time() - t_b
    gsp, gcp = os.path.join(tmpdir, "cfg3_gpu.sbwt"), os.path.join(tmpdir, "cfg3_gpu.tcolors")
    t_b = time.time()
    S.build_colored_index(g.chars, np.cumsum(g.lens).astype(np.uint64), c["k"], gsp, gcp)
    t_gpu_build = time.time() - t_b
    build_same = (open(gsp, "rb").read() == open(sp, "rb").read() and
                  open(gcp, "rb").read() == open(cp, "rb").read())
    chars, ends = T.gen_reads(34, g, args.colors_reads, 1.0, c["read_len"], 0.0,
                              c["read_len"], c["read_len"], c["read_sub"], 0.0)
    t_setup = time.time() - t0
    idx, ci = S.SbwtIndex.open(sp, device=dev), S.ColorIndex.open(cp, device=dev)
    n_reads = len(ends)
    n_k = idx.count_kmers(ends)
    d_chars = torch.from_numpy(chars).to(f"cuda:{dev}")
    d_ends = torch.from_numpy(ends.view(np.int64)).to(f"cuda:{dev}")
    d_res = torch.empty(n_k, dtype=torch.int64, device=f"cuda:{dev}")
    idx.search_reads(d_chars, d_ends, out=d_res)
    # the colors step's input: found indexes per read (+ -1 / -2 counts)
    kpr = n_k // n_reads  # fixed-length reads
    res2 = d_res.view(n_reads, kpr)
    found_mask = (res2 >= 0)
    d_found = d_res[found_mask.view(-1)].contiguous()
    d_offs = torch.zeros(n_reads + 1, dtype=torch.int64, device=f"cuda:{dev}")
    d_offs[1:] = torch.cumsum(found_mask.sum(1), 0)
    d_ids_off = torch.empty(n_reads + 1, dtype=torch.int64, device=f"cuda:{dev}")
    cap = n_reads * 64
    d_ids = torch.empty(cap, dtype=torch.int32, device=f"cuda:{dev}")
    L = S.lib()
    stream = torch.cuda.current_stream(dev)

    def colors_step():
        S.check(L.sbwt_pseudoalign(ci._h, d_found.data_ptr(), d_offs.data_ptr(), None, None,
                                   n_reads, c["tau"], S.DEVICE_POINTERS, d_ids.data_ptr(), cap,
                                   d_ids_off.data_ptr(), stream.cuda_stream))

    for _ in range(2):
        colors_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        colors_step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_col = e0.elapsed_time(e1) / 3 / 1e3
    n_ids = int(d_ids_off[-1].item())
    # parity spot check against the oracle on the first reads
    chk = 2000
    offs_h = d_offs[:chk + 1].cpu().numpy().view(np.uint64)
    found_h = d_found[:int(offs_h[-1])].cpu().numpy().view(np.uint64)
    ids_off_h = d_ids_off[:chk + 1].cpu().numpy()
    ids_h = d_ids[:int(ids_off_h[-1])].cpu().numpy()
    got = [ids_h[ids_off_h[r]:ids_off_h[r + 1]].tolist() for r in range(chk)]
    oc = O.OracleColors(O.ColorsFile.read(cp))
    exp = oc.pseudoalign([found_h[offs_h[r]:offs_h[r + 1]] for r in range(chk)], [0] * chk,
                         [0] * chk, c["tau"])
    # CPU baseline: the restatement on all host threads (OpenMP over reads),
    # on a bounded sample; agreement = per-read id count and id checksum
    n_cpu = min(args.colors_cpu_reads, n_reads)
    offs_c = d_offs[:n_cpu + 1].cpu().numpy().view(np.uint64)
    found_c = d_found[:int(offs_c[-1])].cpu().numpy().view(np.uint64)
    zeros = np.zeros(n_cpu, np.uint64)
    threads = os.cpu_count()
    t1 = time.perf_counter()
    cpu_n, cpu_ck = oc.pseudoalign_mt(found_c, offs_c, zeros, zeros, c["tau"], threads=threads)
    t_cpu = time.perf_counter() - t1
    gio = d_ids_off[:n_cpu + 1].cpu().numpy()
    gids = d_ids[:int(gio[-1])].cpu().numpy().astype(np.uint64)
    gn = np.diff(gio).astype(np.uint64)
    rank_in_read = np.arange(len(gids), dtype=np.uint64) - np.repeat(gio[:-1], gn.astype(np.int64)).astype(np.uint64) + 1
    gck = np.zeros(n_cpu, np.uint64)
    np.add.at(gck, np.repeat(np.arange(n_cpu), gn.astype(np.int64)), (gids + 1) * rank_in_read)
    cpu_agree = bool(np.array_equal(cpu_n, gn) and np.array_equal(cpu_ck, gck))
    # plain colors flow (the reference's ColorSearcher + printer): per batch
    # the R x C counts to the host, then the threshold on the host
    # (ceil((double) size * tau)); timed on a bounded sample
    n_plain = min(args.colors_plain_reads, n_reads)
    pb = min(n_plain, 100_000)
    d_cnt = torch.empty((pb, ci.num_colors), dtype=torch.int32, device=f"cuda:{dev}")
    h_cnt = torch.empty((pb, ci.num_colors), dtype=torch.int32).pin_memory()
    sizes = (d_offs[1:] - d_offs[:-1])[:n_plain].cpu().numpy()
    minimum = np.ceil(sizes.astype(np.float64) * c["tau"]).astype(np.int64)

    def plain_colors():
        n_plain_ids = 0
        for lo in range(0, n_plain, pb):
            m = min(pb, n_plain - lo)
            offs_b = (d_offs[lo:lo + m + 1] - d_offs[lo]).contiguous()
            S.check(L.sbwt_color_counts(ci._h, d_found[int(d_offs[lo].item()):].data_ptr(),
                                        offs_b.data_ptr(), m, d_cnt.data_ptr(),
                                        S.DEVICE_POINTERS, stream.cuda_stream))
            h_cnt[:m].copy_(d_cnt[:m], non_blocking=True)
            torch.cuda.synchronize()
            cnt = h_cnt[:m].numpy()
            mins = minimum[lo:lo + m]
            n_plain_ids += int(((cnt >= mins[:, None]) & (mins[:, None] > 0)).sum())
        return n_plain_ids

    plain_colors()
    t1 = time.perf_counter()
    n_plain_ids = plain_colors()
    t_plain = time.perf_counter() - t1
    e0.record(stream)
    S.check(L.sbwt_pseudoalign(ci._h, d_found.data_ptr(), d_offs.data_ptr(), None, None,
                               n_plain, c["tau"], S.DEVICE_POINTERS, d_ids.data_ptr(), cap,
                               d_ids_off.data_ptr(), stream.cuda_stream))
    fused_ids_h = d_ids_off[n_plain].item()
    e1.record(stream)
    torch.cuda.synchronize()
    t_fused = e0.elapsed_time(e1) / 1e3
    del d_cnt, h_cnt
    colors = {"workload": "2000 genomes x 100 kbp from 8 founders (1-5% divergence), k=31, "
                          f"{n_reads} reads x 150 bp, 0.5% substitutions, tau 0.7",
              "nodes": nodes, "reads": n_reads, "kmers": int(n_k), "ids": n_ids,
              "reads_per_s": n_reads / t_col, "ms_per_step": t_col * 1e3,
              "bit_exact_sample": got == exp, "setup_s": t_setup,
              "colored_build": {"gpu_s": t_gpu_build, "host_s": t_host_build,
                                "host_threads": os.cpu_count(),
                                "files_identical_to_host_build": bool(build_same),
                                "note": "first GPU call of the process, incl. CUDA start-up "
                                        "costs and writing both files"},
              "cpu_baseline": {"value": n_cpu / t_cpu, "unit": "reads/s", "cores": threads,
                               "kind": "port", "sample": f"first {n_cpu} reads (OpenMP "
                               "restatement of d_color_search + d_post_process + the "
                               "threshold, oracle/sbwt_oracle.c)",
                               "agrees_with_gpu": cpu_agree},
              "plain_vs_fused": {
                  "sample_reads": n_plain,
                  "plain_reads_per_s": n_plain / t_plain,
                  "fused_reads_per_s": n_plain / t_fused,
                  "speedup": t_plain / t_fused,
                  "same_id_count": int(n_plain_ids) == int(fused_ids_h),
                  "plain": "the reference's flow: per batch of 100000 reads the R x C counts "
                           "(sbwt_color_counts) copied to the host, threshold on the host",
                  "fused": "sbwt_pseudoalign: counts and threshold on the device, sorted ids"}}
    if args.cli_full:
        try:  # never lets this extra run take the bench line down
            colors["cli_file_to_file"] = colors_cli_file_to_file(sp, cp, chars, ends, c["tau"],
                                                                 tmpdir)
        except Exception as e:  # reported, not raised
            colors["cli_file_to_file"] = {"error": repr(e)}
    del d_res, d_found, d_ids, found_mask, res2
    torch.cuda.empty_cache()
    # fused reads -> colors pipeline from host memory (CUDA graph per batch)
    batch = min(1 << 20, n_reads)
    pipe = S.Pipeline(idx, ci, batch * c["read_len"], batch, tau=c["tau"])
    nb = max(1, min(4, n_reads // batch))
    pipe.run(chars[:int(ends[batch - 1])], ends[:batch], raw=True)
    t1 = time.perf_counter()
    for b in range(nb):
        lo = b * batch
        base = int(ends[lo - 1]) if lo else 0
        pipe.run(chars[base:int(ends[lo + batch - 1])], ends[lo:lo + batch] - base, raw=True)
    t_pipe = time.perf_counter() - t1
    colors["fused_pipeline_reads_per_s"] = nb * batch / t_pipe
    pipe.close()
    # serving loop: Poisson arrivals, log-uniform request sizes in [1, 1e5]
    srv = S.Server(idx, ci, batch_chars=32 << 20, batch_reads=1 << 18, slots=3, tau=c["tau"])
    rng = np.random.default_rng(11)
    serving = {"offline_reads_per_s": colors["fused_pipeline_reads_per_s"], "loads": [],
               "resident": {"colors_workload_sbwt_bytes": int(idx.device_bytes),
                            "index_workload_sbwt_bytes":
                            int(resident_index.device_bytes) if resident_index else 0,
                            "color_index": "resident (sbwt_colors_open)"},
               "admission": "slots open on demand while the device has a slot's bytes free "
                            "above an eighth of its memory (sbwt_server_create)"}
    for offered in (1e5, 1e6, 1e7, 0.8 * colors["fused_pipeline_reads_per_s"]):
        mean_size = (1e5 - 1) / np.log(1e5)
        rate = offered / mean_size
        pending = []
        stop = threading.Event()

        def collector():
            while not stop.is_set() or pending:
                if pending:
                    srv.wait(pending.pop(0), raw=True)
                else:
                    time.sleep(0.0005)

        th = threading.Thread(target=collector)
        th.start()
        srv.stats(reset=True)
        t_start = time.perf_counter()
        t_next = t_start
        while t_next - t_start < args.serve_seconds:
            now = time.perf_counter()
            if now < t_next:
                time.sleep(min(t_next - now, 0.002))
                continue
            size = int(np.exp(rng.uniform(0, np.log(1e5))))
            lo = int(rng.integers(0, n_reads - size))
            base = int(ends[lo - 1]) if lo else 0
            pending.append(srv.submit(chars[base:int(ends[lo + size - 1])],
                                      ends[lo:lo + size] - base))
            t_next += rng.exponential(1.0 / rate)
        t_window = time.perf_counter() - t_start
        stop.set()
        th.join()
        st = srv.stats()
        serving["loads"].append({"slots": srv.slots(), "offered_reads_per_s": offered,
                                 "achieved_reads_per_s": st["reads"] / max(st["elapsed_s"], 1e-9),
                                 "arrival_window_s": t_window, "drain_s": st["elapsed_s"] - t_window,
                                 "p50_ms": st["p50_s"] * 1e3, "p99_ms": st["p99_s"] * 1e3,
                                 "requests": st["requests"], "batches": st["batches"]})
    srv.close()
    return {"colors": colors, "serving": serving}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--reads", type=int, default=CFG["n_reads"])
    ap.add_argument("--presearch", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-sample-reads", type=int, default=500_000)
    ap.add_argument("--index-only", action="store_true",
                    help="skip the batched, colors and serving sections")
    ap.add_argument("--colors-reads", type=int, default=CFG3["n_reads"])
    ap.add_argument("--serve-seconds", type=float, default=3.0)
    ap.add_argument("--colors-cpu-reads", type=int, default=200_000)
    ap.add_argument("--cli-full", action=argparse.BooleanOptionalAction, default=True,
                    help="time the CLI file -> file on all reads of the workload")
    ap.add_argument("--no-full-batched", action="store_true",
                    help="skip the full-size batched workload")
    ap.add_argument("--colors-plain-reads", type=int, default=500_000)
    ap.add_argument("--kernel", type=int, default=-1,
                    help="read search kernel with a k-mer table (sbwt_set_table_kernel): "
                         "0 general, 1 table, 2..5 walks variants, -1 library default")
    ap.add_argument("--colors-only", action="store_true",
                    help="run only the colors and serving sections (profiling runs)")
    ap.add_argument("--cfg1-only", action="store_true",
                    help="run only the 1 Mbp case (profiling runs)")
    ap.add_argument("--gather-sweep", action="store_true",
                    help="print the random-sector gather rate against working-set size "
                         "and exit")
    ap.add_argument("--write-workload", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--seed-reads", type=int, default=1000, help=argparse.SUPPRESS)
    return ap.parse_args()


def profile_file(kernel: str) -> Path:
    """The committed ncu summary of `kernel` on the 1 M-read case."""
    return REPO / "profiles" / f"{kernel}_100Mbp_1Mreads_full.md"


def profiled_traffic_per_kmer(kernel: str):
    """DRAM bytes (read + write) per k-mer of the search kernel from the
    committed ncu capture of the 1 M-read case; traffic grows with the k-mers
    processed, so it scales to a full launch by the k-mer count."""
    p = profile_file(kernel)
    try:
        for ln in p.read_text().splitlines():
            if ln.startswith("traffic_bytes_per_kmer:"):
                return float(ln.split(":")[1])
    except OSError:
        pass
    return None


def link_roofline(torch, dev, h2d_bytes, d2h_bytes, step_s):
    """The host link's bound on an e2e step: pinned H2D and D2H copy rates of
    this GPU measured on 1 GiB (CUDA events, best of 3), and the step's
    minimum time if the two directions overlap fully (the larger of the two
    transfer times), over the measured step time."""
    n = 1 << 30
    d = torch.empty(n, dtype=torch.uint8, device=f"cuda:{dev}")
    h = torch.empty(n, dtype=torch.uint8).pin_memory()
    rates = {}
    for name, dst, src in (("h2d", d, h), ("d2h", h, d)):
        best = 0.0
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            best = max(best, n / (e0.elapsed_time(e1) / 1e3))
        rates[name] = best
    del d, h
    t_min = max(h2d_bytes / rates["h2d"], d2h_bytes / rates["d2h"])
    return {"h2d_gbs": rates["h2d"] / 1e9, "d2h_gbs": rates["d2h"] / 1e9,
            "t_min_ms": t_min * 1e3, "frac": t_min / step_s,
            "how": "cudaMemcpyAsync of 1 GiB between pinned host memory and the device, "
                   "best of 3; t_min = max(H2D bytes / H2D rate, D2H bytes / D2H rate)"}


def load_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, dev: int):
        self.dev = dev
        self.proc = None
        self.rows = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        for ln in out.strip().splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 7:
                self.rows.append(f)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def make_workload(seed_reads: int, n_reads: int, tmpdir: str):
    import sbwt_tools as T
    c = CFG
    g = T.gen_genomes(20240601, c["n_genomes"], c["genome_len"], c["n_founders"],
                      c["sub"], c["sub"], c["indel"])
    path = os.path.join(tmpdir, "cfg2.sbwt")
    nodes = T.build_sbwt(g, c["k"], path)
    chars, ends = T.gen_reads(seed_reads, g, n_reads, 1.0, c["len_median"],
                              c["len_sigma"], c["len_min"], c["len_max"],
                              c["read_sub"], c["n_rate"])
    return g, path, nodes, chars, ends


def kmer_count(ends: np.ndarray, k: int) -> int:
    lens = np.diff(np.concatenate([[0], ends.astype(np.int64)]))
    return int(np.maximum(lens - k + 1, 0).sum())


def index_config(args, world: int, nodes: int, n_kmers: int, n_chars: int) -> dict:
    """The `config` of the index-search line, the same for both arms."""
    return {"workload": "index search: 100 Mbp reference (40 x 2.5 Mbp genomes "
                        "from 4 founders, 2% subs, 0.1% indels), k=31, both strands; "
                        f"{args.reads} reads log-normal length (median 150, 31-1000), "
                        "0.5% subs, 0.1% N", "k": CFG["k"], "nodes": int(nodes),
            "reads_per_gpu": args.reads, "kmers_per_gpu": int(n_kmers),
            "chars_per_gpu": int(n_chars), "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (no flush needed)"}


def workload_files(seed_reads: int, n_reads: int, sample_reads: int, tmpdir: str):
    """The index workload for the reference arm, made in a child process (the
    project's generator and builder stay out of the reference arm's process):
    the .sbwt path and the first `sample_reads` reads (chars, ends)."""
    subprocess.run([sys.executable, str(Path(__file__).resolve()), "--write-workload", tmpdir,
                    "--reads", str(n_reads), "--cpu-sample-reads", str(sample_reads),
                    "--seed-reads", str(seed_reads)], check=True)
    chars = np.load(os.path.join(tmpdir, "sample_chars.npy"))
    ends = np.load(os.path.join(tmpdir, "sample_ends.npy"))
    with open(os.path.join(tmpdir, "meta.json")) as f:
        meta = json.load(f)
    return os.path.join(tmpdir, "cfg2.sbwt"), chars, ends, meta


def write_workload(args):
    """Child side of workload_files."""
    g, path, nodes, chars, ends = make_workload(args.seed_reads, args.reads,
                                                args.write_workload)
    n = min(args.cpu_sample_reads, len(ends))
    np.save(os.path.join(args.write_workload, "sample_chars.npy"), chars[:int(ends[n - 1])])
    np.save(os.path.join(args.write_workload, "sample_ends.npy"), ends[:n])
    with open(os.path.join(args.write_workload, "meta.json"), "w") as f:
        json.dump({"nodes": int(nodes), "kmers": kmer_count(ends, CFG["k"]),
                   "chars": int(ends[-1])}, f)


def gather_sweep(S, dev):
    """Random 32-byte-sector gather rate against the working-set size: for
    buffers of 32 MB .. 8 GB and 1, 4 and 8 independent dependent-load
    chains per thread (2048 threads per SM), sbwt_measure_random_sectors;
    the implied loaded latency is threads x chains / rate.  The read search
    looks up random sectors in working sets of these sizes, so this curve is
    its ceiling."""
    import torch
    L = S.lib()
    L.sbwt_measure_random_sectors.argtypes = [C.c_int, C.c_uint64, C.c_int,
                                              C.POINTER(C.c_double), C.POINTER(C.c_double)]
    threads = torch.cuda.get_device_properties(dev).multi_processor_count * 2048
    rows = []
    for mb in (32, 64, 128, 256, 512, 1024, 2048, 4096, 8192):
        row = {"bytes": mb << 20}
        for chains in (1, 4, 8):
            gbs, sps = C.c_double(), C.c_double()
            S.check(L.sbwt_measure_random_sectors(dev, mb << 20, chains, C.byref(gbs),
                                                  C.byref(sps)))
            row[f"gsectors_s_{chains}"] = sps.value / 1e9
            row[f"latency_us_{chains}"] = threads * chains / sps.value * 1e6
        rows.append(row)
    return {"gather_sweep": rows, "threads": threads}


def random_sector_peak(S, dev, ws_bytes):
    """Measured random 32-byte-sector gather rate (sectors/s) of this GPU over
    a buffer of ws_bytes (the search kernels' roofline denominator): best of
    4 and 8 independent dependent-load chains per thread."""
    L = S.lib()
    L.sbwt_measure_random_sectors.argtypes = [C.c_int, C.c_uint64, C.c_int,
                                              C.POINTER(C.c_double), C.POINTER(C.c_double)]
    best = 0.0
    for chains in (4, 8):
        gbs, sps = C.c_double(), C.c_double()
        S.check(L.sbwt_measure_random_sectors(dev, int(ws_bytes), chains, C.byref(gbs),
                                              C.byref(sps)))
        best = max(best, sps.value)
    return best


KERNELS = {0: "search_reads_kernel", 1: "search_table_kernel", 2: "search_walks_kernel",
           3: "search_walks_kernel", 4: "search_walks_kernel", 5: "search_walks_kernel",
           6: "search_kmers_kernel", 8: "search_walks_kernel", 9: "search_walks_kernel",
           10: "search_walks_kernel", 11: "search_kmers_kernel", 12: "search_kmers_kernel",
           13: "search_walks_kernel", 14: "search_walks_kernel", 15: "search_kmers_seq_kernel",
           16: "search_walks_kernel", 17: "search_walks_kernel", 18: "search_walks_kernel",
           19: "search_kmers_kernel"}
DEFAULT_KERNEL_MODE = 7
KMERS_KERNEL_MAX_BYTES = 256 << 20  # mode 7 picks the k-mers kernel up to this


def search_kernel_name(idx, mode: int) -> str:
    """The read search kernel that runs for `mode` (sbwt_set_table_kernel) on
    an index: without a k-mer table always the general kernel."""
    mode = DEFAULT_KERNEL_MODE if mode < 0 else mode
    table = idx.set_kmer_table(True)
    if not table:
        return KERNELS[0]
    if mode == 7:
        mode = 11 if 0 < idx.filter_bytes() and table + idx.filter_bytes() <= \
            KMERS_KERNEL_MAX_BYTES else 17
    return KERNELS[mode]


FILTER_KERNELS = ("search_walks_kernel", "search_kmers_kernel", "search_kmers_seq_kernel")


def index_working_sets(idx):
    """Bytes the read search touches at random: the rank blocks of the four
    vectors plus the suffix-group-start words (every step); the table it
    starts a k-mer from (one lookup per k-mer not reached by a stream step):
    the k-mer table when the index has one, else the presearch level; and
    the k-mer filter in front of the table (10 bits per k-mer)."""
    n = idx.num_bits
    hot = 4 * (n // 192 + 1) * 32 + (n + 63) // 64 * 8
    table = idx.set_kmer_table(True)  # its size (kept when present)
    if table:
        return hot, table, idx.filter_bytes()
    entry = 8 if n < (1 << 32) else 16
    return hot, (4 ** idx.presearch_letters) * entry, 0


def sector_roofline(S, dev, idx, n_hot, n_pre, kernel_s, n_filter=0, cold=False):
    """Random-sector roofline of the read search: the time the kernel's
    sectors take at the measured random-gather rate of their own working set
    (rank blocks + group words; the k-mer table or presearch level; the
    k-mer filter), over the kernel time.  The rates are those of a warm L2
    (the microbenchmark repeats its gathers over one buffer).  cold=True
    (L2 flushed before the timed launch) adds `cold_l2`: each class's
    expected distinct sectors, S * (1 - exp(-n / S)) for n uniform random
    loads over S sectors, are first touches served by DRAM at the measured
    rate of a 2 GiB buffer; the rest at the class's warm rate."""
    hot_b, pre_b, filt_b = index_working_sets(idx)
    r_hot = random_sector_peak(S, dev, hot_b)
    r_pre = random_sector_peak(S, dev, pre_b)
    r_filt = random_sector_peak(S, dev, filt_b) if (filt_b and n_filter) else 0.0
    t_min = n_hot / r_hot + n_pre / r_pre + (n_filter / r_filt if r_filt else 0.0)
    cold_l2 = None
    if cold:
        r_dram = random_sector_peak(S, dev, 2 << 30)
        t_cold, first = 0.0, {}
        for name, n, ws, r in (("hot", n_hot, hot_b, r_hot), ("lookup", n_pre, pre_b, r_pre),
                               ("filter", n_filter, filt_b, r_filt)):
            if not n or not r:
                continue
            secs = max(1.0, ws / 32)
            d = secs * -math.expm1(-n / secs)
            first[name] = int(d)
            t_cold += d / r_dram + (n - d) / r
        cold_l2 = {"frac": t_cold / kernel_s, "t_min_ms": t_cold * 1e3,
                   "dram_peak_gsectors_s": r_dram / 1e9, "first_touch_sectors": first,
                   "model": "L2 flushed before the launch: a sector's first touch comes "
                            "from DRAM (random-sector rate of a 2 GiB buffer), later "
                            "touches at the working set's warm rate"}
    out = {"frac": t_min / kernel_s, "t_min_ms": t_min * 1e3, "kernel_ms": kernel_s * 1e3,
           "achieved_gsectors_s": (n_hot + n_pre + n_filter) / kernel_s / 1e9,
           "hot": {"sectors": int(n_hot), "working_set_bytes": int(hot_b),
                   "peak_gsectors_s": r_hot / 1e9},
           "lookup": {"sectors": int(n_pre), "working_set_bytes": int(pre_b),
                      "peak_gsectors_s": r_pre / 1e9},
           "peak_source": "sbwt_measure_random_sectors over buffers of each working set's "
                          "size, best of 4/8 chains"}
    if n_filter:
        out["filter"] = {"sectors": int(n_filter), "working_set_bytes": int(filt_b),
                         "peak_gsectors_s": r_filt / 1e9}
    if cold_l2 is not None:
        out["cold_l2"] = cold_l2
    return out


def bench_cfg1(args, S, torch, dev, tmpdir):
    """The CPU-comparable case: 1 Mbp i.i.d. genome, k=31, both strands;
    100,000 reads x 150 bp, half sampled from the genome with 1% substitutions
    and half i.i.d. random.  L2 is flushed before every timed step.  Reports
    k-mers/s, the search kernel's random-sector rate against the measured
    random-sector roofline at the index's size, and the reference's own CPU
    build on all reads."""
    import sbwt_tools as T
    L = S.lib()
    g = T.gen_genomes(1, 1, 1_000_000)
    path = os.path.join(tmpdir, "cfg1.sbwt")
    nodes = T.build_sbwt(g, 31, path)
    chars, ends = T.gen_reads(2, g, 100_000, 0.5, 150, 0.0, 150, 150, 0.01, 0.0)
    idx = S.SbwtIndex.open(path, device=dev)
    nk = idx.count_kmers(ends)
    d_chars = torch.from_numpy(chars).to(f"cuda:{dev}")
    d_ends = torch.from_numpy(ends.view(np.int64)).to(f"cuda:{dev}")
    d_out = torch.empty(nk, dtype=torch.int64, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)

    def step():
        idx.search_reads(d_chars, d_ends, out=d_out, stream=stream.cuda_stream)

    L.sbwt_profile_enable(1, 1)
    step()
    torch.cuda.synchronize()
    ctr = (C.c_uint64 * 16)()
    L.sbwt_profile_read(None, None, None, ctr)
    L.sbwt_profile_enable(0, 0)
    kernel = search_kernel_name(idx, args.kernel)
    n_filter = int(ctr[3]) if kernel in FILTER_KERNELS else 0
    sectors = int(ctr[0]) + int(ctr[1]) + int(ctr[2]) + n_filter
    for _ in range(max(3, args.warmup)):
        step()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    L.sbwt_profile_enable(1, 0)
    total_ms, n_steps = 0.0, max(5, args.steps)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(n_steps):
        flush.zero_()
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
    kms, kl, _ = C.c_double(), C.c_uint64(), C.c_uint64()
    L.sbwt_profile_read(C.byref(kms), C.byref(kl), None, None)
    L.sbwt_profile_enable(0, 0)
    kern_s = kms.value / max(1, kl.value) / 1e3
    out_h = d_out.cpu().numpy()
    res = {"workload": "1 Mbp i.i.d. genome, k=31, both strands; 100000 reads x 150 bp, "
                       "50% from the genome (1% substitutions), 50% random",
           "nodes": nodes, "reads": len(ends), "kmers": int(nk),
           "found_frac": float((out_h >= 0).mean()),
           "kmers_per_s": nk / (total_ms / n_steps / 1e3), "ms_per_step": total_ms / n_steps,
           "l2": "flushed (256 MB write) before every timed step",
           "kernel": kernel,
           "random_sector": dict(sector_roofline(S, dev, idx, int(ctr[1]) + int(ctr[2]),
                                                 int(ctr[0]), kern_s, n_filter, cold=True),
                                 sectors_per_kmer=sectors / nk)}
    r = cpu_reference_rate(path, chars, ends, 31, len(ends))
    if r is not None:
        rate, nkc, dt, threads, (bits, pos, ref) = r
        res["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads,
                               "kind": "reference", "sample": f"all {len(ends)} reads"}
        res["bit_exact_vs_cpu_reference"] = bool(np.array_equal(idx.search(bits, pos), ref))
    idx.close()
    return res


def fastq_text(chars, ends):
    """Reads as FASTQ records ("@r", sequence, "+", quality 'I'), vectorised."""
    lens = np.diff(np.concatenate([[0], ends.astype(np.int64)]))
    rec = 3 + lens + 1 + 2 + lens + 1
    start = np.concatenate([[0], np.cumsum(rec)[:-1]])
    out = np.full(int(rec.sum()), ord("I"), dtype=np.uint8)
    for off, b in ((0, b"@"), (1, b"r"), (2, b"\n")):
        out[start + off] = b[0]
    seq_at = start + 3
    idx = np.repeat(seq_at - np.concatenate([[0], ends[:-1].astype(np.int64)]), lens) + \
        np.arange(int(lens.sum()))
    out[idx] = chars[:int(lens.sum())]
    out[seq_at + lens] = ord("\n")
    out[seq_at + lens + 1] = ord("+")
    out[seq_at + lens + 2] = ord("\n")
    out[start + rec - 1] = ord("\n")
    return out


def bench_io(args, S, torch, dev, tmpdir, idx, path, chars, ends, d_out, d_ends, n_kmers):
    """The reads' ends of the path on the GPU: FASTQ parsing (sbwt_fastx_parse)
    against the host reader, ascii formatting of the timed run's results
    (sbwt_format_index_results) against the host writer, and the command line
    tool end to end on one FASTQ file."""
    import subprocess
    L = S.lib()
    L.sbwt_fastx_read.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
    L.sbwt_free.argtypes = [C.c_void_p]
    L.sbwt_write_index_results.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_uint64, C.c_uint32]
    stream = torch.cuda.current_stream(dev)
    out = {}
    # parsing: 2 M reads as FASTQ
    n_sub = min(2_000_000, len(ends))
    sub_ends = ends[:n_sub]
    text = fastq_text(chars, sub_ends)
    fq = os.path.join(tmpdir, "q.fq")
    text.tofile(fq)
    d_text = torch.from_numpy(text).to(f"cuda:{dev}")
    n_chars = int(sub_ends[-1])
    d_pc = torch.empty(n_chars, dtype=torch.uint8, device=f"cuda:{dev}")
    d_pe = torch.empty(n_sub, dtype=torch.int64, device=f"cuda:{dev}")
    nc, nr = C.c_uint64(), C.c_uint64()

    def parse():
        S.check(L.sbwt_fastx_parse(d_text.data_ptr(), len(text), d_pc.data_ptr(), n_chars,
                                   d_pe.data_ptr(), n_sub, C.byref(nc), C.byref(nr),
                                   S.DEVICE_POINTERS, dev, stream.cuda_stream))

    parse()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        parse()
    e1.record(stream)
    torch.cuda.synchronize()
    t_dev = e0.elapsed_time(e1) / 3 / 1e3
    exact = (nr.value == n_sub and np.array_equal(d_pe.cpu().numpy().view(np.uint64), sub_ends)
             and np.array_equal(d_pc.cpu().numpy(), chars[:n_chars]))
    ch, en, hc, hr = C.c_void_p(), C.c_void_p(), C.c_uint64(), C.c_uint64()
    t0 = time.perf_counter()
    S.check(L.sbwt_fastx_read(fq.encode(), C.byref(ch), C.byref(hc), C.byref(en), C.byref(hr)))
    t_host = time.perf_counter() - t0
    L.sbwt_free(ch)
    L.sbwt_free(en)
    out["parse"] = {"input": f"{n_sub} reads as FASTQ ({len(text)} bytes), device-resident",
                    "device_gb_s": len(text) / t_dev / 1e9, "device_ms": t_dev * 1e3,
                    "host_reader_gb_s": len(text) / t_host / 1e9, "host_threads": 1,
                    "speedup": t_host / t_dev, "exact_vs_input": bool(exact)}
    del d_text, d_pc, d_pe
    # formatting the timed run's results (all reads, ascii)
    nb = C.c_uint64()
    fmt_args = (d_out.data_ptr(), d_ends.data_ptr(), len(ends), CFG["k"], 0)
    rc = L.sbwt_format_index_results(*fmt_args, None, 0, C.byref(nb), S.DEVICE_POINTERS, dev,
                                     stream.cuda_stream)
    assert rc == S.E_CAPACITY, rc
    d_fmt = torch.empty(nb.value, dtype=torch.uint8, device=f"cuda:{dev}")

    def fmt():
        S.check(L.sbwt_format_index_results(*fmt_args, d_fmt.data_ptr(), nb.value, C.byref(nb),
                                            S.DEVICE_POINTERS, dev, stream.cuda_stream))

    fmt()
    e0.record(stream)
    for _ in range(3):
        fmt()
    e1.record(stream)
    torch.cuda.synchronize()
    t_fmt = e0.elapsed_time(e1) / 3 / 1e3
    # the host writer on the first 2 M reads, and the bytes compared
    n_sk = int(np.maximum(np.diff(np.concatenate([[0], sub_ends.astype(np.int64)])) -
                          CFG["k"] + 1, 0).sum())
    h_res = d_out[:n_sk].cpu().numpy().view(np.uint64)
    t0 = time.perf_counter()
    S.check(L.sbwt_write_index_results(os.path.join(tmpdir, "hw").encode(), 0, 0,
                                       h_res.ctypes.data, sub_ends.ctypes.data, n_sub,
                                       CFG["k"]))
    t_hw = time.perf_counter() - t0
    host_bytes = open(os.path.join(tmpdir, "hw.txt"), "rb").read()
    same = d_fmt[:len(host_bytes)].cpu().numpy().tobytes() == host_bytes
    out["format_ascii"] = {"kmers": int(n_kmers), "bytes": int(nb.value),
                           "device_ms": t_fmt * 1e3, "device_kmers_per_s": n_kmers / t_fmt,
                           "device_gb_s_written": nb.value / t_fmt / 1e9,
                           "host_writer_kmers_per_s": n_sk / t_hw, "host_threads": 1,
                           "sample_bytes_equal_host_writer": bool(same)}
    del d_fmt
    torch.cuda.empty_cache()
    # the command line tool on the FASTQ file (index load + device path)
    cli = REPO / "sbwt-search_b200" / "_build" / "sbwt_search"
    t0 = time.perf_counter()
    r = subprocess.run([str(cli), "index", "-i", path, "-q", fq, "-o",
                        os.path.join(tmpdir, "cli"), "--no-headers"], capture_output=True)
    t_cli = time.perf_counter() - t0
    cli_same = r.returncode == 0 and open(os.path.join(tmpdir, "cli.txt"), "rb").read() == host_bytes
    out["cli"] = {"command": "sbwt_search index -i <cfg2.sbwt> -q <2M-read FASTQ> -o <prefix> "
                             "--no-headers", "wall_s": t_cli, "kmers": n_sk,
                  "kmers_per_s_incl_index_load": n_sk / t_cli,
                  "output_equal_host_writer": bool(cli_same), "rc": r.returncode}
    if args.cli_full:
        # file -> file on all reads of the workload: the FASTQ written in
        # pieces, the CLI once on an empty query (process start, index load:
        # rank blocks, presearch pyramid, k-mer table and filter) and once on
        # the full query; the difference is the search itself, file to file
        full = os.path.join(tmpdir, "full.fq")
        with open(full, "wb") as f:
            for lo in range(0, len(ends), 1_000_000):
                hi = min(len(ends), lo + 1_000_000)
                base = int(ends[lo - 1]) if lo else 0
                f.write(fastq_text(chars[base:int(ends[hi - 1])], ends[lo:hi] - base).tobytes())
        empty = os.path.join(tmpdir, "empty.fq")
        open(empty, "wb").close()
        fq_bytes = os.path.getsize(full)
        t0 = time.perf_counter()
        r0 = subprocess.run([str(cli), "index", "-i", path, "-q", empty, "-o",
                             os.path.join(tmpdir, "cli_empty"), "--no-headers"],
                            capture_output=True)
        t_load = time.perf_counter() - t0
        t0 = time.perf_counter()
        r1 = subprocess.run([str(cli), "index", "-i", path, "-q", full, "-o",
                             os.path.join(tmpdir, "cli_full"), "--no-headers"],
                            capture_output=True)
        t_all = time.perf_counter() - t0
        out_bytes = os.path.getsize(os.path.join(tmpdir, "cli_full.txt")) if r1.returncode == 0 \
            else 0
        try:
            os.remove(os.path.join(tmpdir, "cli_full.txt"))
        except OSError:
            pass
        # the same with the bool print mode (1 byte per k-mer: less to write)
        t0 = time.perf_counter()
        r2 = subprocess.run([str(cli), "index", "-i", path, "-q", full, "-o",
                             os.path.join(tmpdir, "cli_bool"), "--no-headers", "-p", "bool"],
                            capture_output=True)
        t_bool = time.perf_counter() - t0
        # the same two runs with the query and the outputs in RAM-backed
        # /dev/shm (when it has the room): the file system out of the way
        shm = None
        try:
            st = os.statvfs("/dev/shm")
            room = st.f_bavail * st.f_frsize
        except OSError:
            room = 0
        if room > fq_bytes + 3 * max(out_bytes, 1) + (4 << 30):
            d = tempfile.mkdtemp(dir="/dev/shm")
            try:  # never lets this extra run take the bench line down
                q = os.path.join(d, "full.fq")
                with open(full, "rb") as src, open(q, "wb") as dst:
                    while True:
                        b = src.read(1 << 28)
                        if not b:
                            break
                        dst.write(b)
                t0 = time.perf_counter()
                s1 = subprocess.run([str(cli), "index", "-i", path, "-q", q, "-o",
                                     os.path.join(d, "out"), "--no-headers"],
                                    capture_output=True)
                t_s1 = time.perf_counter() - t0
                same_size = s1.returncode == 0 and \
                    os.path.getsize(os.path.join(d, "out.txt")) == out_bytes
                try:
                    os.remove(os.path.join(d, "out.txt"))
                except OSError:
                    pass
                t0 = time.perf_counter()
                s2 = subprocess.run([str(cli), "index", "-i", path, "-q", q, "-o",
                                     os.path.join(d, "outb"), "--no-headers", "-p", "bool"],
                                    capture_output=True)
                t_s2 = time.perf_counter() - t0
                shm = {"where": "query and outputs in /dev/shm (RAM-backed)",
                       "rc": [s1.returncode, s2.returncode], "wall_s": t_s1,
                       "kmers_per_s_file_to_file": n_kmers / max(t_s1 - t_load, 1e-9),
                       "kmers_per_s_incl_index_load": n_kmers / t_s1,
                       "output_bytes_equal_disk_run": bool(same_size),
                       "bool_print_mode": {"wall_s": t_s2, "kmers_per_s_file_to_file":
                                           n_kmers / max(t_s2 - t_load, 1e-9)}}
            except Exception as e:  # reported, not raised
                shm = {"error": repr(e)}
            finally:
                for x in ("full.fq", "out.txt", "outb.bool"):
                    try:
                        os.remove(os.path.join(d, x))
                    except OSError:
                        pass
                try:
                    os.rmdir(d)
                except OSError:
                    pass
        for x in ("full.fq", "cli_bool.bool"):
            try:
                os.remove(os.path.join(tmpdir, x))
            except OSError:
                pass
        out["cli_full"] = {
            "command": "sbwt_search index -i <cfg2.sbwt> -q <all reads as FASTQ> -o <prefix> "
                       "--no-headers (ascii output)",
            "reads": int(len(ends)), "kmers": int(n_kmers), "fastq_bytes": int(fq_bytes),
            "output_bytes": int(out_bytes), "rc": [r0.returncode, r1.returncode],
            "wall_s": t_all, "index_load_and_start_s": t_load,
            "kmers_per_s_file_to_file": n_kmers / max(t_all - t_load, 1e-9),
            "kmers_per_s_incl_index_load": n_kmers / t_all,
            "bool_print_mode": {"rc": r2.returncode, "wall_s": t_bool,
                                "kmers_per_s_file_to_file":
                                    n_kmers / max(t_bool - t_load, 1e-9)},
            "ram_files": shm}
    return out


def bench_build(S, T, g, host_path, tmpdir):
    """The 100 Mbp index built on the GPU (sbwt_build_index) against the host
    builder (all host threads), and the two files compared byte for byte."""
    import torch
    ends = np.cumsum(g.lens).astype(np.uint64)
    gpu_path = os.path.join(tmpdir, "cfg2_gpu.sbwt")
    S.build_index((g.chars, ends), CFG["k"], gpu_path)  # warm (CUDA context, caches)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nodes = S.build_index((g.chars, ends), CFG["k"], gpu_path)
    t_gpu = time.perf_counter() - t0
    host2 = os.path.join(tmpdir, "cfg2_host.sbwt")
    t0 = time.perf_counter()
    T.build_sbwt(g, CFG["k"], host2)
    t_host = time.perf_counter() - t0
    same = open(gpu_path, "rb").read() == open(host_path, "rb").read()
    return {"input": f"{len(g.lens)} genomes, {int(ends[-1])} bp, k={CFG['k']}, both strands",
            "nodes": int(nodes), "gpu_s": t_gpu, "host_s": t_host,
            "host_threads": os.cpu_count(), "speedup": t_host / t_gpu,
            "file_identical_to_host_build": bool(same),
            "note": "wall time incl. host<->device copies and writing the .sbwt file"}


def dist_setup(args):
    import replicas as R
    world, rank, local = R.world()
    if world > 1 and args.impl == "ours":
        import torch
        torch.cuda.set_device(local)
    pg = R.init("nccl" if args.impl == "ours" else "gloo", timeout_s=900)
    return world, rank, local, pg


def cpu_reference_rate(path, chars, ends, k, sample_reads):
    """SBWT-Search's own index kernels compiled for the host (oracle/_ref),
    all host threads, on the first `sample_reads` reads.  Returns
    (k-mers/s, k-mers, seconds, threads, results)."""
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    L = O.ref_lib()
    if L is None:
        return None
    sb = O.SbwtFile.read(path)
    idx = O.OracleIndex(sb.acgt, sb.num_bits, sb.k, use_ref=True)
    n = min(sample_reads, len(ends))
    sub_ends = ends[:n]
    sub_chars = chars[:int(sub_ends[-1])]
    bits, _ = O.seq_to_bits(sub_chars.tobytes())
    pos = O.positions_of(sub_ends, k)
    threads = L.ref_max_threads()
    idx.search_positions(bits, pos[:1000], threads=threads)  # warm
    t0 = time.perf_counter()
    res = idx.search_positions(bits, pos, threads=threads)
    dt = time.perf_counter() - t0
    return len(pos) / dt, len(pos), dt, threads, (bits, pos, res)


def run_reference(args, world, rank, local, pg):
    """--impl reference: the reference's own CPU implementation of the index
    step (oracle/_ref), timed per step on a bounded sample of the workload."""
    if rank != 0:
        return
    with tempfile.TemporaryDirectory() as d:
        path, chars, ends, meta = workload_files(1000 + rank, args.reads,
                                                 args.cpu_sample_reads, d)
        times, last = [], None
        for i in range(args.warmup + args.steps):
            r = cpu_reference_rate(path, chars, ends, CFG["k"], args.cpu_sample_reads)
            if r is None:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "oracle/_ref (reference kernels built for the host) missing"}))
                return
            if i >= args.warmup:
                times.append(r[2])
                last = r
        rate, nk, dt, threads, _ = last
        med = statistics.median(times)
        value = nk / med
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": med * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u64", "data": "synthetic (seeded; generated at start-up)", "impl": "reference",
                "config": index_config(args, world, meta["nodes"], meta["kmers"],
                                       meta["chars"]),
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                                 "kind": "reference",
                                 "sample": f"first {args.cpu_sample_reads} reads "
                                           f"({nk} k-mers) per step"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.write_workload:
        write_workload(args)
        return
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank, local, pg)
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()
        return
    import torch
    import sbwt_b200 as S
    torch.cuda.set_device(local)
    dev = local
    if args.gather_sweep or args.colors_only or args.cfg1_only:
        if rank == 0:
            if args.gather_sweep:
                print(json.dumps(gather_sweep(S, dev)), flush=True)
            elif args.cfg1_only:
                S.set_table_kernel(args.kernel)
                with tempfile.TemporaryDirectory() as d:
                    print(json.dumps(bench_cfg1(args, S, torch, dev, d)), flush=True)
            else:
                with tempfile.TemporaryDirectory() as d:
                    print(json.dumps(bench_colors_and_serving(args, S, torch, dev, d, rank)),
                          flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    S.set_table_kernel(args.kernel)
    L = S.lib()
    L.sbwt_profile_enable.argtypes = [C.c_int, C.c_int]
    L.sbwt_profile_read.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    tmp = tempfile.TemporaryDirectory()
    t0 = time.time()
    g, path, nodes, chars, ends = make_workload(1000 + rank, args.reads, tmp.name)
    t_gen = time.time() - t0
    idx = S.SbwtIndex.open(path, device=dev, presearch_letters=args.presearch)
    n_kmers = idx.count_kmers(ends)
    n_chars = int(ends[-1])
    # device-resident inputs (larger than L2: 1.7 GB chars, 11 GB results)
    d_chars = torch.from_numpy(chars).to(f"cuda:{dev}")
    d_ends = torch.from_numpy(ends.view(np.int64)).to(f"cuda:{dev}")
    d_out = torch.empty(n_kmers, dtype=torch.int64, device=f"cuda:{dev}")
    stream = torch.cuda.current_stream(dev)

    def step_dev():
        n = idx.search_reads(d_chars, d_ends, out=d_out, stream=stream.cuda_stream)
        assert n == n_kmers

    # one counting pass (outside the timed region): work per k-mer
    L.sbwt_profile_enable(1, 1)
    step_dev()
    torch.cuda.synchronize()
    ctr = (C.c_uint64 * 16)()
    L.sbwt_profile_read(None, None, None, ctr)
    n_pre, n_block, n_sg, n_probe = (int(ctr[0]), int(ctr[1]), int(ctr[2]), int(ctr[3]))
    n_iter, n_lane, n_known, n_searched = (int(ctr[4]), int(ctr[5]), int(ctr[6]), int(ctr[7]))
    L.sbwt_profile_enable(0, 0)

    for _ in range(args.warmup):
        step_dev()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    L.sbwt_profile_enable(1, 0)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step_dev()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    search_ms, search_launches, launches = C.c_double(), C.c_uint64(), C.c_uint64()
    L.sbwt_profile_read(C.byref(search_ms), C.byref(search_launches), C.byref(launches),
                        None)
    L.sbwt_profile_enable(0, 0)
    import replicas as R
    ms = R.max_over_ranks(pg, ms, device=f"cuda:{dev}")  # slowest rank
    ms_step = ms / args.steps
    value = n_kmers * world / (ms_step / 1e3)

    # parity spot check of the timed output against the oracle (small sample)
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O
    out_host = d_out[:200_000].cpu().numpy().view(np.uint64)

    # e2e through the host-pointer C ABI call from pinned memory
    e2e = None
    if not args.no_e2e:
        h_chars = torch.from_numpy(chars).pin_memory()
        h_ends = torch.from_numpy(ends.view(np.int64)).pin_memory()
        h_out = torch.empty(n_kmers, dtype=torch.int64).pin_memory()
        hc, he, ho = h_chars.numpy(), h_ends.numpy().view(np.uint64), h_out.numpy().view(np.uint64)
        idx.search_reads(hc, he, out=ho)  # warm
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        e_steps = max(1, min(args.steps, 3))
        for _ in range(e_steps):
            idx.search_reads(hc, he, out=ho)
        e_dt = (time.perf_counter() - t0) / e_steps
        e_dt = R.max_over_ranks(pg, e_dt, device=f"cuda:{dev}")
        assert np.array_equal(ho[:200_000], out_host), "e2e output differs from device path"
        e2e = {"value": n_kmers * world / e_dt, "unit": UNIT,
               "h2d_bytes_per_step": int(chars.nbytes + ends.nbytes),
               "d2h_bytes_per_step": int(n_kmers * 8),
               "ms_per_step": e_dt * 1e3,
               "results": "u64 per k-mer, DMA into pinned host memory",
               "link": link_roofline(torch, dev, chars.nbytes + ends.nbytes, n_kmers * 8,
                                     e_dt)}
        del h_chars, h_ends, h_out

    # roofline of the dominant kernel (the read search kernel)
    peak, peak_kind = load_peaks()
    kern_ms = search_ms.value / max(1, search_launches.value)
    # the kernel that ran: with the k-mer table (k <= 31) the walks kernel by
    # default, else the general kernel
    kernel = search_kernel_name(idx, args.kernel)
    n_filter = n_probe if kernel in FILTER_KERNELS else 0
    if n_filter:
        n_probe = 0
    # algorithmic bytes per launch (what this kernel's algorithm must move):
    # one 32-byte sector per k-mer-table or presearch lookup, per k-mer filter
    # word, per rank block and per suffix-group word the search reads; 8 B
    # result per k-mer; 2 bits of packed input + 1 invalid bit per char.
    alg_bytes = ((n_pre + n_block + n_sg + n_filter) * 32 + n_kmers * 8 + n_chars / 4 +
                 n_chars / 8)
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    traffic_pk = profiled_traffic_per_kmer(kernel)
    try:
        rs = sector_roofline(S, dev, idx, n_block + n_sg, n_pre, kern_ms / 1e3, n_filter)
    except Exception as e:  # reported as unmeasured, never hides the headline
        rs = {"error": repr(e)}

    extra = {}
    if not args.index_only and rank == 0:  # per-GPU sections: rank 0 only
        torch.cuda.empty_cache()
        try:
            import sbwt_tools as T
            extra["build"] = bench_build(S, T, g, path, tmp.name)
        except Exception as e:
            extra["build"] = {"error": repr(e)}
        try:
            extra["io"] = bench_io(args, S, torch, dev, tmp.name, idx, path, chars, ends, d_out,
                                   d_ends, n_kmers)
        except Exception as e:
            extra["io"] = {"error": repr(e)}
        try:
            extra["cfg1"] = bench_cfg1(args, S, torch, dev, tmp.name)
        except Exception as e:
            extra["cfg1"] = {"error": repr(e)}
        try:
            extra["batched_small_files"] = bench_batched(args, idx, S, torch, dev, d_out)
        except Exception as e:  # reported, never hides the headline
            extra["batched_small_files"] = {"error": repr(e)}
        del d_out, d_chars, d_ends
        torch.cuda.empty_cache()
        if not args.no_full_batched:
            try:
                extra["batched"] = bench_batched_full(args, idx, S, torch, dev)
            except Exception as e:  # reported, never hides the headline
                extra["batched"] = {"error": repr(e)}
            torch.cuda.empty_cache()
        try:
            extra.update(bench_colors_and_serving(args, S, torch, dev, tmp.name, rank,
                                                  resident_index=idx))
        except Exception as e:
            extra["colors"] = {"error": repr(e)}

    cpu = None
    if rank == 0 and not args.no_cpu:
        r = cpu_reference_rate(path, chars, ends, CFG["k"], args.cpu_sample_reads)
        if r is not None:
            rate, nk, dt, threads, (bits, pos, res) = r
            got = idx.search(bits, pos)
            agree = bool(np.array_equal(got, res))
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"first {args.cpu_sample_reads} reads ({nk} k-mers), "
                             f"SBWT-Search's own d_search/d_presearch built for the "
                             f"host, OpenMP", "bit_exact_vs_gpu": agree}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded; generated at start-up)",
        "config": index_config(args, world, nodes, n_kmers, n_chars),
        "launch": {"presearch_letters": idx.presearch_letters,
                   "kernel_mode": args.kernel if args.kernel >= 0 else DEFAULT_KERNEL_MODE,
                   "kernels": f"{kernel}"
                              + (" (the default, automatic mode 7 picks it for this index)"
                                 if args.kernel < 0 else f" (mode {args.kernel})")
                              + ", grid of 8 x 256-thread blocks per SM, tiles of "
                                "k-mers / (resident threads x 8) rounded up to 16 slots, "
                                "16 to 128"},
        "gpu_launches": int(launches.value),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": (None if traffic_pk is None else traffic_pk * n_kmers),
                     "traffic_source": "ncu capture of the 1 M-read case scaled by k-mers "
                                       f"({profile_file(kernel).relative_to(REPO)})",
                     "peak_kind": peak_kind, "kernel": kernel,
                     "kernel_ms": kern_ms,
                     "work": {"table_or_presearch_lookups": n_pre,
                              "rank_block_sectors": n_block,
                              "suffix_group_words": n_sg, "probe_iterations": n_probe,
                              "filter_words": n_filter,
                              "bytes_per_kmer": alg_bytes / n_kmers,
                              "warp_iterations": n_iter,
                              "lanes_loading_per_iteration": n_lane / max(n_iter, 1),
                              "kmers_written_without_search": n_known,
                              "kmers_searched": n_searched,
                              "lane_steps_by_path": dict(zip(
                                  ["stream", "filter" if n_filter else "presearch", "walk",
                                   "group_scan", "kmer_table", "probe"],
                                  [int(x) for x in ctr[8:14]])),
                              "distinct_paths_per_iteration": int(ctr[14]) / max(n_iter, 1)},
                     "random_sector": rs},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clk.summary(),
        "setup_s": t_gen,
    }
    line.update(extra)
    if rank == 0:
        print(json.dumps(line), flush=True)
    idx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
