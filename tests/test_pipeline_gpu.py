"""Batched pipelines (one CUDA graph per batch, persistent search launch with
a device work queue) and the continuous-batching server: results are
identical to the single calls, alone and in a mix of concurrent requests."""
import threading

import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
import sbwt_tools as T
from helpers import TMP, mixed_reads, oracle_index, oracle_results, synthetic

pytestmark = pytest.mark.gpu


def colored(seed=5, n=150, length=800, founders=6):
    g = T.gen_genomes(seed, n, length, founders, 0.01, 0.05, 0.0)
    sp = TMP / f"pcol_{seed}_{n}_{length}.sbwt"
    cp = TMP / f"pcol_{seed}_{n}_{length}.tcolors"
    T.build_colored(g, 31, str(sp), str(cp))
    return g, str(sp), str(cp)


def test_pipeline_index_mode_matches_search_reads():
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    p = S.Pipeline(idx, None, 1 << 20, 20000)
    for seed, n in ((1, 3000), (2, 50), (3, 0), (4, 7000), (5, 1)):
        chars, ends = mixed_reads(g, seed, n, sub=0.01, n_rate=0.005)
        got = p.run(chars, ends)
        assert np.array_equal(got, idx.search_reads(chars, ends))
        assert np.array_equal(got, oracle_results(oracle_index(path, 8), chars, ends))


def test_pipeline_colors_mode_matches_two_step_calls():
    g, sp, cp = colored()
    idx, ci = S.SbwtIndex.open(sp), S.ColorIndex.open(cp)
    p = S.Pipeline(idx, ci, 1 << 20, 20000, tau=0.7)
    oc = O.OracleColors(O.ColorsFile.read(cp))
    for seed, n in ((11, 800), (12, 3), (13, 2000)):
        chars, ends = T.gen_reads(seed, g, n, 0.9, 120, 0.4, 20, 400, 0.01, 0.003)
        got = p.run(chars, ends)
        res = idx.search_reads(chars, ends)
        per, t = [], 0
        for r in T.split_reads(chars, ends):
            m = max(0, len(r) - 30)
            per.append(res[t:t + m])
            t += m
        found = [x[x < O.INVALID] for x in per]
        assert got == oc.pseudoalign(found, [0] * len(per), [0] * len(per), 0.7)


def test_pipeline_rejects_oversized_batch():
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    p = S.Pipeline(S.SbwtIndex.open(path), None, 1000, 10)
    chars, ends = mixed_reads(g, 1, 100)
    with pytest.raises(S.SbwtError) as e:
        p.run(chars, ends)
    assert e.value.code == S.E_INVALID


def _requests(g, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = int(np.exp(rng.uniform(0, np.log(3000))))
        out.append(T.gen_reads(seed * 1000 + i, g, size, 0.9, 150, 0.0, 150, 150, 0.005, 0.0))
    return out


def test_server_colors_same_alone_and_in_mix():
    g, sp, cp = colored()
    idx, ci = S.SbwtIndex.open(sp), S.ColorIndex.open(cp)
    srv = S.Server(idx, ci, batch_chars=200_000, batch_reads=1500, slots=3, tau=0.7)
    reqs = _requests(g, 40, 3)
    alone = []
    for chars, ends in reqs[:5]:  # one at a time
        alone.append(srv.wait(srv.submit(chars, ends)))
    ids = [None] * len(reqs)

    def client(lo, hi):
        rids = [(i, srv.submit(*reqs[i])) for i in range(lo, hi)]
        for i, rid in rids:
            ids[i] = srv.wait(rid)

    th = [threading.Thread(target=client, args=(i, i + 10)) for i in range(0, 40, 10)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert ids[:5] == alone  # same alone and in the mix
    p = S.Pipeline(idx, ci, 1 << 22, 1 << 16, tau=0.7)
    for i in range(len(reqs)):  # and the same as one direct batch
        assert ids[i] == p.run(*reqs[i])
    st = srv.stats()
    assert st["requests"] >= 45 and st["p99_s"] >= st["p50_s"] > 0
    srv.close()


def test_server_index_mode_splits_large_requests():
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    srv = S.Server(idx, None, batch_chars=20_000, batch_reads=200, slots=2)
    chars, ends = mixed_reads(g, 9, 2500, sub=0.01, n_rate=0.005)  # ~13 batches
    vals, offs = srv.wait(srv.submit(chars, ends))
    assert np.array_equal(vals, idx.search_reads(chars, ends))
    assert offs[-1] == len(vals) and len(offs) == len(ends) + 1
    empty = srv.wait(srv.submit(b"", np.zeros(0, np.uint64)))
    assert len(empty[0]) == 0
    srv.close()


def test_server_admits_slots_by_free_device_memory():
    """A slot opens only while the device keeps a slot's bytes free above an
    eighth of its memory: with room, all slots open at creation; with that
    room taken by another allocation only the first opens, waiting batches
    find no room (the refusals are counted) and requests still complete on
    it with the results of direct calls; once the memory is back, slots open
    again as batches wait."""
    import torch
    g, sp, cp = colored()
    idx, ci = S.SbwtIndex.open(sp), S.ColorIndex.open(cp)
    reqs = _requests(g, 24, 5)
    p = S.Pipeline(idx, ci, 1 << 22, 1 << 16, tau=0.7)
    exp = [p.run(*r) for r in reqs]
    srv = S.Server(idx, ci, batch_chars=200_000, batch_reads=1500, slots=4, tau=0.7)
    info = srv.slots()
    assert info["open"] == 4 and info["slot_bytes"] > 0
    srv.close()
    free, total = torch.cuda.mem_get_info()
    keep = total // 8 + info["slot_bytes"] // 2  # less than a slot above the reserve
    hog = torch.empty(max(free - keep, 0), dtype=torch.uint8, device="cuda")
    try:
        srv = S.Server(idx, ci, batch_chars=200_000, batch_reads=1500, slots=4, tau=0.7)
        assert srv.slots()["open"] == 1
        got = [srv.wait(rid) for rid in [srv.submit(*r) for r in reqs]]
        assert got == exp
        after = srv.slots()
        assert after["open"] == 1 and after["denied"] > 0
    finally:
        del hog
        torch.cuda.empty_cache()
    got = [srv.wait(rid) for rid in [srv.submit(*r) for r in reqs]]
    assert got == exp
    assert 1 <= srv.slots()["open"] <= 4
    srv.close()
