"""Replica sharding across GPUs (one process per GPU, torch.distributed).

The per-timestep path has no collective: replicas are independent, so a run
over several GPUs only partitions them and reduces timings at the end.

* weak scaling: every rank advances its own seeded ensemble of the same size
  (seed + 1000 * rank), so per-GPU work is fixed as ranks are added;
* strong scaling: one ensemble is split by greedy longest-processing-time
  assignment over the O(N^2) far-field cost, sum over replicas of N_r^2.

Timings are taken on each rank with CUDA events and combined as the maximum
over ranks (the job finishes with its slowest rank).
"""
from __future__ import annotations

import heapq


def lpt_partition(costs: list[float], nranks: int) -> list[list[int]]:
    """Greedy LPT: replicas in decreasing cost, each to the least-loaded rank
    (ties to the lowest rank).  Returns, per rank, its replica indices in
    ascending order."""
    heap = [(0.0, r) for r in range(nranks)]
    parts: list[list[int]] = [[] for _ in range(nranks)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def replica_cost(system) -> float:
    """Relative cost of one step: the far-field pairs dominate, N^2."""
    n = system.Np
    return float(n * n)


def rank_systems(systems: list, rank: int, world: int) -> list:
    """This rank's share of one ensemble (strong scaling)."""
    if world <= 1:
        return list(systems)
    parts = lpt_partition([replica_cost(s) for s in systems], world)
    return [systems[i] for i in parts[rank]]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank float over the process group (value itself when
    torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
