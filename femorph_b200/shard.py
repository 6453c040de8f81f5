"""Placing independent solves on GPUs (one process per GPU).

The explicit-flow path shards by problem: batched and served solves are
independent, so each rank owns a subset of the problems and no data-path
collective is needed.  The only cross-rank operations are the host-side
assignment (identical on every rank, no communication) and the reduction of
timings / counters for reporting.
"""
from __future__ import annotations

import heapq


def assign(costs, world: int):
    """Longest-processing-time assignment of problems to `world` ranks.

    costs: per-problem work (e.g. elements x steps).  Returns a list with the
    rank of every problem.  Deterministic (ties broken by problem index, then
    rank), so every rank computes the same assignment without communicating.
    """
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return owner


def mine(costs, world: int, rank: int):
    """Indices of the problems rank `rank` owns."""
    return [i for i, r in enumerate(assign(costs, world)) if r == rank]


def reduce_max(value: float, dist=None, device=None) -> float:
    """Max over ranks of a per-rank time (the step time of a job is the
    slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, dist=None, device=None) -> float:
    """Sum over ranks of a per-rank counter (element-steps done)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
