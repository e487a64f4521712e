"""Multi-GPU plumbing for batches of independent matrices.

The matrices of a batch are independent, so a batch shards across ranks
with no exchange step: each rank (one process per GPU) solves its own
slice, and only timing / status is combined.  Nothing here touches the data
path; torch.distributed carries the scalar reductions.
"""
from __future__ import annotations

import heapq


def shard_range(L: int, rank: int, world: int):
    """Contiguous slice (start, count) of a uniform batch of L matrices for
    `rank` of `world`; the first L % world ranks take one extra matrix."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, rem = divmod(L, world)
    start = rank * base + min(rank, rem)
    return start, base + (1 if rank < rem else 0)


def shard_uneven(ns, world: int):
    """Cost-balanced partition of an uneven batch: matrix sizes `ns`, cost
    proportional to n^3, greedy longest-processing-time.  Returns one list of
    matrix indices per rank (each list in ascending index order)."""
    order = sorted(range(len(ns)), key=lambda i: -int(ns[i]) ** 3)
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(ns[i]) ** 3, r))
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, device=None):
    """Max of a per-rank scalar (elapsed device time) over the default
    process group; the identity when torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
