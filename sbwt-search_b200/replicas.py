"""Multi-GPU plumbing for the search: index replicas, no data-path collective.

Every k-mer walk and every read's color merge is independent, so N GPUs run N
replicas of the read-only index, each searching its own share of the reads
(one process per GPU, launched by torchrun).  The only collectives are the
timing ones: a barrier around the timed region and the maximum of the
per-rank elapsed times (the job is as slow as its slowest rank).
"""
from __future__ import annotations

import datetime
import os


def world():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 600.0):
    """Initialises the default process group when world_size > 1 (rendezvous
    from MASTER_ADDR / MASTER_PORT); returns torch.distributed or None."""
    n, _, _ = world()
    if n <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def shard(n_items: int, rank: int, world_size: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of n_items for `rank` (sizes differ by <= 1)."""
    q, r = divmod(n_items, world_size)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def max_over_ranks(dist, value: float, device=None) -> float:
    """The maximum of `value` over all ranks (identity without a group)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value: float, device=None) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
