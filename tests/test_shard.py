"""CPU, world size 2 over gloo: instance sharding assigns every instance to
exactly one rank, balances load, and gathers results in the original order.
The per-rank thinning here is the oracle (the kernels need a GPU); the code
under test is the sharding and gathering host logic."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from begputhinning_b200.shard import assign
from tests.helpers import blobs2d, blobs3d


def test_assign_balances_and_covers():
    sizes = [100, 90, 80, 10, 10, 10, 5, 5, 1]
    shards = assign(sizes, 3)
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(sizes)
    assert assign(sizes, 1) == [list(range(len(sizes)))]


def _items():
    rng = np.random.default_rng(3)
    return [blobs2d(rng, 40 + 9 * k, 50 + 7 * k, 4) for k in range(7)] + [blobs3d(rng, 12, 14, 16, 2)]


def _thin(batch):
    from oracle import pyoracle as po
    return [po.thin2d(x)[0] if x.ndim == 2 else po.thin3d(x)[0] for x in batch]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from begputhinning_b200.shard import run_sharded
        res = run_sharded(_items(), _thin)
        if rank == 0:
            want = _thin(_items())
            q.put(all(np.array_equal(a, b) for a, b in zip(res, want)) and len(res) == len(want))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.timeout(120)
def test_two_rank_gloo_sharding():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok = q.get(timeout=100)
    for p in procs:
        p.join(timeout=60)
    assert ok
    assert all(p.exitcode == 0 for p in procs)
