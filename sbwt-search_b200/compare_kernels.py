"""Times the two read search kernels on the index workload and checks that
their outputs are equal.

    python sbwt-search_b200/compare_kernels.py [--reads N] [--lib PATH]

Builds the 100 Mbp index workload of bench.py (first N reads, default 10 M),
opens the index (k-mer table included), and for the general kernel and then
the table kernel (sbwt_set_table_kernel 0, 1): one counting pass, 3 warm-up
passes and 5 timed passes of sbwt_search_reads over device-resident inputs.
Prints one JSON line: per kernel the pass time, the kernel time (CUDA events
on its stream) and the work counters; and whether the outputs are equal.
"""
import argparse
import ctypes as C
import json
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reads", type=int, default=10_000_000)
    ap.add_argument("--lib", default=None,
                    help="another build of libsbwt_b200.so (default: _build/)")
    args = ap.parse_args()
    import numpy as np
    import torch
    import bench
    import sbwt_b200 as S
    if args.lib:
        S.LIB_PATH = Path(args.lib).resolve()
    L = S.lib()
    L.sbwt_profile_enable.argtypes = [C.c_int, C.c_int]
    L.sbwt_profile_read.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    tmp = tempfile.TemporaryDirectory()
    _, path, _, chars, ends = bench.make_workload(1000, args.reads, tmp.name)
    idx = S.SbwtIndex.open(path, device=0)
    n_k = idx.count_kmers(ends)
    d_chars = torch.from_numpy(chars).cuda()
    d_ends = torch.from_numpy(ends.view(np.int64)).cuda()
    outs, res = {}, {"kmers": n_k, "lib": str(S.LIB_PATH)}
    for name, tk in (("general", False), ("table", True)):
        S.set_table_kernel(tk)
        out = torch.empty(n_k, dtype=torch.int64, device="cuda")
        L.sbwt_profile_enable(1, 1)
        idx.search_reads(d_chars, d_ends, out=out)
        torch.cuda.synchronize()
        ctr = (C.c_uint64 * 16)()
        L.sbwt_profile_read(None, None, None, ctr)
        L.sbwt_profile_enable(0, 0)
        for _ in range(3):
            idx.search_reads(d_chars, d_ends, out=out)
        torch.cuda.synchronize()
        L.sbwt_profile_enable(1, 0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            idx.search_reads(d_chars, d_ends, out=out)
        e1.record()
        torch.cuda.synchronize()
        sm, sl = C.c_double(), C.c_uint64()
        L.sbwt_profile_read(C.byref(sm), C.byref(sl), None, None)
        L.sbwt_profile_enable(0, 0)
        res[name] = {"pass_ms": e0.elapsed_time(e1) / 5,
                     "kernel_ms": sm.value / max(1, sl.value), "counters": list(ctr)}
        outs[name] = out
    S.set_table_kernel(True)
    res["equal"] = bool(torch.equal(outs["general"], outs["table"]))
    print(json.dumps(res), flush=True)
    if not res["equal"]:
        sys.exit(1)


if __name__ == "__main__":
    main()
