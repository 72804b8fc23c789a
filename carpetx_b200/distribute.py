"""Distribution of a refinement level's boxes over ranks, one process per GPU.

In CarpetX a new or regridded level arrives with a BoxArray and an AMReX
DistributionMapping (CarpetX/src/driver.cxx:1244-1256, MakeNewLevelFromCoarse
receiving `ba` and `dm`); every process then prolongates only the boxes it
owns, from coarse data already copied next to them.  The transfer therefore
shards by box with no exchange between ranks on the data path: a rank's part
of the level is just a LevelPlan over its own boxes.

The mapping here is a knapsack one, like AMReX's knapsack distribution
strategy: boxes are weighted by their work (fine points x components) and
dealt, the heaviest first, to the least-loaded rank (ties to the lower rank),
the longest-processing-time rule (makespan at most 4/3 of the optimum).
It is a pure function of the box list, so every rank computes the same
mapping without communicating.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def box_cost(fine_lo: Sequence[int], fine_hi: Sequence[int], ncomp: int) -> int:
    """Work of one box: fine points of the fine box times components."""
    n = 1
    for d in range(3):
        n *= max(0, int(fine_hi[d]) - int(fine_lo[d]) + 1)
    return n * int(ncomp)


def knapsack(costs: Sequence[int], nranks: int) -> list[int]:
    """Owner rank of each box: heaviest first to the least-loaded rank."""
    if nranks < 1:
        raise ValueError("nranks must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    heap = [(0, r) for r in range(nranks)]
    owner = [0] * len(costs)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + int(costs[i]), r))
    return owner


def rank_loads(costs: Sequence[int], owner: Sequence[int], nranks: int) -> list[int]:
    loads = [0] * nranks
    for c, r in zip(costs, owner):
        loads[r] += int(c)
    return loads


def my_boxes(boxes: Sequence, costs: Sequence[int], rank: int, world: int) -> list:
    """The boxes rank `rank` of `world` owns, in their original order."""
    owner = knapsack(costs, world)
    return [b for b, r in zip(boxes, owner) if r == rank]


def max_over_ranks(x: float, device=None) -> float:
    """Maximum of a per-rank number over the default process group (the
    identity without one); `device` is where the reduction tensor lives
    (a CUDA device for NCCL, the CPU for gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    """Sum of a per-rank number over the default process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
