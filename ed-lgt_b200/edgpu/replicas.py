"""Instance sharding across ranks (one process per GPU).

The instances of a sweep (couplings, charge sectors, quench runs) are
independent, so they are split across ranks with no data-path collective:
each rank solves its shard; only results and timings are gathered.
Assignment is greedy longest-processing-time on an estimated cost (sector
dimension times mean row length), deterministic for a given cost list.
"""

from __future__ import annotations

import numpy as np

__all__ = ["shard_instances", "gather_objects", "max_over_ranks"]


def shard_instances(costs, world_size: int, rank: int) -> list[int]:
    """Indices of the instances rank ``rank`` solves."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("need 0 <= rank < world_size")
    costs = np.asarray(costs, dtype=float)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world_size)
    owner = np.empty(len(costs), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return [int(i) for i in np.nonzero(owner == rank)[0]]


def gather_objects(obj, world_size: int):
    """All-gather of picklable per-rank results (list indexed by rank)."""
    if world_size == 1:
        return [obj]
    import torch.distributed as dist

    out = [None] * world_size
    dist.all_gather_object(out, obj)
    return out


def max_over_ranks(x: float, world_size: int, device=None) -> float:
    if world_size == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
