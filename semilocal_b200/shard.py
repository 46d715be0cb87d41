"""Pair sharding over ranks (one process per GPU).

Pairs are independent, so a batch shards by pair with no exchange on the data path: each rank combs its
own pairs and keeps its braids.  The partition is a cost-balanced greedy (longest processing time first over
the cells m*n); the only collectives are the host-side bookkeeping below (timing max over ranks, optional
gathering of small per-pair results).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def shard_pairs(costs: Sequence[int], world: int) -> List[List[int]]:
    """Indices of the pairs each of `world` ranks takes: pairs in decreasing cost, each to the rank with the
    least cost so far (ties to the lower rank).  Every index appears exactly once; each rank's list is in
    increasing index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    heap = [(0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(costs[i]), r))
    return [sorted(s) for s in shards]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of a per-rank value (a step time) over all ranks; the value itself without a process
    group."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_scores(scores, dist=None, dst: int = 0):
    """Per-rank lists of (pair index, score) gathered on rank dst (None on the other ranks)."""
    if dist is None or not dist.is_initialized():
        return [list(scores)]
    out = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(list(scores), out, dst=dst)
    return out
