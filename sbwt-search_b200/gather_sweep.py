"""Random 32-byte-sector gather rate of one GPU against the working-set size.

    python sbwt-search_b200/gather_sweep.py [--device D]

For buffers from 32 MB to 8 GB and 1, 4 and 8 independent dependent-load
chains per thread (2048 threads per SM), runs sbwt_measure_random_sectors
and prints one JSON line: sectors/s per size and chain count, and the
implied loaded latency (threads x chains / rate).  The read search kernels
look up random sectors in working sets of these sizes (rank blocks ~91 MB,
k-mer table 4 GiB, presearch level 2 GiB on the 100 Mbp index), so this
curve is their ceiling.
"""
import argparse
import ctypes as C
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    import sbwt_b200 as S
    L = S.lib()
    L.sbwt_measure_random_sectors.argtypes = [C.c_int, C.c_uint64, C.c_int,
                                              C.POINTER(C.c_double), C.POINTER(C.c_double)]
    sms = 148
    try:
        import torch
        sms = torch.cuda.get_device_properties(args.device).multi_processor_count
    except Exception:
        pass
    threads = sms * 2048
    rows = []
    for mb in (32, 64, 128, 256, 512, 1024, 2048, 4096, 8192):
        row = {"bytes": mb << 20}
        for chains in (1, 4, 8):
            gbs, sps = C.c_double(), C.c_double()
            S.check(L.sbwt_measure_random_sectors(args.device, mb << 20, chains,
                                                  C.byref(gbs), C.byref(sps)))
            row[f"gsectors_s_{chains}"] = sps.value / 1e9
            row[f"latency_us_{chains}"] = threads * chains / sps.value * 1e6
        rows.append(row)
    print(json.dumps({"device": args.device, "threads": threads, "sweep": rows}), flush=True)


if __name__ == "__main__":
    main()
