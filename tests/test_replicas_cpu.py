"""The N > 1 path's host logic on CPU: two gloo ranks shard a read batch,
search it with the CPU oracle (standing in for each rank's GPU replica),
and reduce the timing with max-over-ranks; the union of the shards equals
the single-process result."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import replicas as R


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import sys
    from pathlib import Path
    repo = Path(__file__).resolve().parents[1]
    for p in (str(repo / "tests"), str(repo / "oracle"), str(repo / "sbwt-search_b200")):
        sys.path.insert(0, p)
    from helpers import synthetic, oracle_index, mixed_reads, oracle_results
    dist = R.init("gloo", timeout_s=60)
    n, r, _ = R.world()
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    chars, ends = mixed_reads(g, 3, 1000)
    lo, hi = R.shard(len(ends), r, n)
    base = int(ends[lo - 1]) if lo else 0
    part = oracle_results(oracle_index(path, 8), chars[base:int(ends[hi - 1])],
                          ends[lo:hi] - base)
    np.save(os.path.join(out_dir, f"part{r}.npy"), part)
    t = R.max_over_ranks(dist, float(r + 1))
    tot = R.sum_over_ranks(dist, float(len(part)))
    np.save(os.path.join(out_dir, f"red{r}.npy"), np.array([t, tot]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    from helpers import synthetic, oracle_index, mixed_reads, oracle_results
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    chars, ends = mixed_reads(g, 3, 1000)
    full = oracle_results(oracle_index(path, 8), chars, ends)
    parts = [np.load(tmp_path / f"part{r}.npy") for r in range(2)]
    assert np.array_equal(np.concatenate(parts), full)
    for r in range(2):
        t, tot = np.load(tmp_path / f"red{r}.npy")
        assert t == 2.0 and tot == len(full)


def test_shard_covers_everything():
    for n in (0, 1, 7, 1000):
        for w in (1, 2, 3, 8):
            spans = [R.shard(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
