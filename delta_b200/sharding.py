"""Multi-GPU plumbing: one process per GPU, work split without data exchange.

The pair list and the candidate body pairs are independent work items, so N ranks take
disjoint contiguous shards and no collective is needed on the data path (the reference's
distributed driver exchanges ghost triangles because it decomposes space,
zoltan/migration.cpp:1020-1284; a pair list needs no such exchange).  The only
collective is the max-over-ranks of the timings.
"""
from __future__ import annotations


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [lo, hi) share of n items for `rank` of `world` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()
