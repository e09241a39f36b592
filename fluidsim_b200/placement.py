"""Placement of independent grids on the GPUs of one node.

Batched and served grids never exchange data: each grid lives whole on one GPU and the ranks
share nothing on the hot path. Placement is a deterministic bin packing that every rank computes
identically from the same list, so no collective is needed to agree on it; the only collectives
are the host-side timing and metric reductions below.
"""
from __future__ import annotations

from typing import List, Sequence


def place(costs: Sequence[float], sizes: Sequence[int], world: int, budget: int) -> List[int]:
    """Rank of every grid: longest-processing-time-first by cost (cells, the work per step),
    each grid to the least-loaded rank whose device bytes stay within budget. Ties go to the
    lower rank, so every rank computes the same answer. Raises ValueError when a grid fits no
    rank."""
    if world <= 0:
        raise ValueError("world must be positive")
    if len(costs) != len(sizes):
        raise ValueError("costs and sizes differ in length")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    used = [0] * world
    rank = [-1] * len(costs)
    for i in order:
        candidates = [r for r in range(world) if used[r] + sizes[i] <= budget]
        if not candidates:
            raise ValueError(f"grid {i} ({sizes[i]} bytes) fits no rank within {budget} bytes")
        r = min(candidates, key=lambda c: (load[c], c))
        rank[i] = r
        load[r] += costs[i]
        used[r] += sizes[i]
    return rank


def mine(assignment: Sequence[int], rank: int) -> List[int]:
    """Indices placed on `rank`, in their original order."""
    return [i for i, r in enumerate(assignment) if r == rank]


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (timings are reported as the slowest rank's)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
