"""Replicas across GPUs: one process per GPU, each running its own ensemble
members, with no collective on the data path.

Ensemble members are independent solves, so an ensemble spreads over GPUs by
members (the reference spreads samples over MPI sub-communicators,
src/azeban.cpp:131-152).  The only communication is host-side bookkeeping:
which members a rank runs, and the max over ranks of a timed region (the
whole job is as slow as its slowest rank).  Works with any torch.distributed
backend: NCCL on GPUs, gloo on CPU (the tests).
"""

from __future__ import annotations

import heapq
from typing import Sequence


def partition_by_cost(costs: Sequence[float], world: int) -> list[list[int]]:
    """Members (indices into `costs`) for each of `world` ranks: largest cost
    first, each to the rank with the least cost so far (ties to the lowest
    rank), so every rank's total stays within one member's cost of the
    others'.  Every member lands on exactly one rank; a rank's list is in
    ascending member order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def _reduce(x: float, op_name: str, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    dev = device
    if dev is None:
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x: float, device=None) -> float:
    """Max of x over all ranks (x itself without a process group)."""
    return _reduce(x, "MAX", device)


def sum_over_ranks(x: float, device=None) -> float:
    """Sum of x over all ranks (x itself without a process group)."""
    return _reduce(x, "SUM", device)


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def aggregate_rate(units_per_rank: float, world: int, slowest_ms: float) -> float:
    """Whole-job rate: the units every rank processed, over the slowest
    rank's time (weak scaling: each rank runs the same amount of work)."""
    if slowest_ms <= 0:
        raise ValueError("time must be positive")
    return world * units_per_rank / (slowest_ms / 1e3)
