"""Test helper for the multi-process path (tests/test_sharding.py): one rank's share of
a pair list solved on the CPU by the oracle (test infrastructure only), plus the
max-over-ranks of a timing, over whatever process group is initialised."""
from __future__ import annotations

import time


def run_shard(rank: int, world: int, n: int = 3000, seed: int = 5):
    from oracle.oracle import Oracle

    from delta_b200.scenarios import narrowphase_pairs
    from delta_b200.sharding import max_over_ranks, shard_range

    a, b, _, _ = narrowphase_pairs(n, seed)
    lo, hi = shard_range(n, rank, world)
    o = Oracle()
    t0 = time.perf_counter()
    _, _, d, _ = o.pairs(0, a[:, lo:hi], b[:, lo:hi], nthreads=1)
    t = time.perf_counter() - t0 + 0.001 * rank
    full = o.pairs(0, a, b, nthreads=1)[2] if rank == 0 else None
    (mx,) = max_over_ranks([t])
    return {"dist": d, "time": t, "max_time": mx, "full": full}
