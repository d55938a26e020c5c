"""Placement of docking work across ranks (one process per GPU).

Complexes never exchange data with one another in REMC docking (replica
exchange happens inside a complex's own temperature ladder), so the path
shards with no collective on its data: each rank takes a disjoint set of
complexes and only timings and counters are reduced.  Complexes are placed by
longest-processing-time first on their cost (replicas x ligand atoms x
protein points per MC step), so the ranks finish at about the same time.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def complex_cost(n_rep: int, lna: int, pnp: int) -> float:
    """Pair evaluations of one MC step of a complex's replicas."""
    return float(n_rep) * float(lna) * float(pnp)


def place(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Indices of the complexes of each rank: costliest first onto the rank
    with the least work so far (ties by rank), each rank's list ascending."""
    if world_size < 1:
        raise ValueError(f"world_size={world_size}")
    heap = [(0.0, r) for r in range(world_size)]
    out: list[list[int]] = [[] for _ in range(world_size)]
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(x) for x in out]


def my_items(costs: Sequence[float], world_size: int, rank: int) -> list[int]:
    if not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside [0, {world_size})")
    return place(costs, world_size)[rank]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank value (device time of the slowest rank) through
    torch.distributed (NCCL on GPUs, gloo on CPU); the value itself when no
    process group is initialised."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    """Sum of a per-rank counter (replica-MC-steps done) over the ranks."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
