"""Multi-GPU: instances are independent, so a job shards by instance with no
collective on the data path.  One process per GPU (torchrun); each rank
thins its shard with its own batch engine; results are gathered only when a
caller asks for them on one rank.

``assign`` balances shards by voxel count (longest-processing-time-first:
instances in decreasing size, each to the currently lightest rank).
"""
from __future__ import annotations

import heapq


def assign(sizes, world: int):
    """Shard indices for each rank, balancing total size."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + sizes[i], r))
    for s in shards:
        s.sort()
    return shards


def run_sharded(items, thin_fn, gather: bool = True):
    """Thin this rank's shard of `items` with `thin_fn(list_of_arrays) ->
    list_of_arrays`; with gather, rank 0 receives every result in the
    original order (torch.distributed must be initialised; any backend)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(), dist.get_world_size()
    mine = assign([it.size for it in items], world)[rank]
    outs = thin_fn([items[i] for i in mine])
    if not gather:
        return dict(zip(mine, outs))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(list(zip(mine, outs)), gathered, dst=0)
    if rank != 0:
        return None
    result = [None] * len(items)
    for part in gathered:
        for i, o in part:
            if result[i] is not None:
                raise RuntimeError(f"instance {i} thinned by two ranks")
            result[i] = o
    if any(r is None for r in result):
        raise RuntimeError("an instance was not assigned to any rank")
    return result
