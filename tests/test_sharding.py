"""N>1 host logic on CPU: shard ranges cover the pair list exactly once, and the
max-over-ranks reduction works across a 2-rank gloo group."""
import os

import numpy as np
import pytest

from delta_b200.sharding import shard_range


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (10, 3), (1 << 20, 8), (7, 7)])
def test_shards_partition_the_range(n, world):
    seen = np.zeros(n, np.int64)
    for r in range(world):
        lo, hi = shard_range(n, r, world)
        assert 0 <= lo <= hi <= n
        seen[lo:hi] += 1
    assert np.all(seen == 1)


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from tests.shard_helper import run_shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, run_shard(rank, world)))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shards_and_max():
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    # each rank solved its own shard with the oracle; together they equal the whole list
    assert res[0]["max_time"] == res[1]["max_time"] == max(res[0]["time"], res[1]["time"])
    d = np.concatenate([res[0]["dist"], res[1]["dist"]])
    assert np.array_equal(d, res[0]["full"])
