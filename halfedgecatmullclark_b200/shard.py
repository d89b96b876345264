"""Sharding of independent cages over ranks (one process per GPU).

Refinement of one cage never reads another cage's data, so a batch of cages
shards with no exchange at all: each rank refines its own cages (a ``Batch``
on its own GPU) and the only collective is the max of the ranks' device times
when a job is timed.  The assignment is computed identically on every rank
from the cages' sizes, so no rank has to broadcast it.

Work model: the refined halfedges of a cage (sum over depths 1..D), which the
level kernels' time follows.
"""
from __future__ import annotations

import heapq

import numpy as np


def cage_work(cage, depth: int) -> int:
    """Refined halfedges of depths 1..depth (4^d H0 each)."""
    return int(sum(cage.H * 4 ** d for d in range(1, depth + 1)))


def shard(work: list[int], world: int) -> list[list[int]]:
    """Cage indices per rank: longest work first onto the least-loaded rank
    (ties broken by rank), each rank's list in increasing cage order.  The
    largest load is at most 4/3 of the optimum (Graham's LPT bound)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(work)), key=lambda i: (-int(work[i]), i))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(work[i]), r))
    return [sorted(x) for x in out]


def loads(work: list[int], parts: list[list[int]]) -> np.ndarray:
    return np.array([sum(int(work[i]) for i in p) for p in parts], dtype=np.int64)


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """Max of a per-rank scalar (a device time) over the process group."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
