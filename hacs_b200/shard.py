"""Sharding of the batched job stream across ranks (one process per GPU).

Jobs of the stream are independent units (a GEMM and a rank each), so N GPUs
split them with no data-path collective: every rank computes the same
deterministic assignment from the jobs' shapes, runs its share through the
batched entry points on its own GPU, and the ranks of all jobs are gathered on
the host in job order.  The reference has no multi-device job stream; its
tape splits work across host threads by tile (src/Engine/Passes.cpp:617-800).
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np


def job_cost(m, n, k) -> np.ndarray:
    """Predicted work of GEMM (m x k by k x n) followed by rank(C), in modMAC:
    m*n*k for the product plus m*n*min(m, n) for the elimination."""
    m = np.asarray(m, dtype=np.float64)
    n = np.asarray(n, dtype=np.float64)
    k = np.asarray(k, dtype=np.float64)
    return m * n * k + m * n * np.minimum(m, n)


def shard_jobs(costs: Sequence[float], world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment: jobs by decreasing cost (ties by
    index), each to the least-loaded rank (ties by rank).  Deterministic, so all
    ranks agree without communication.  Each rank's list is in job order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda j: (-costs[j], j))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for j in order:
        load, r = heapq.heappop(heap)
        out[r].append(j)
        heapq.heappush(heap, (load + float(costs[j]), r))
    for lst in out:
        lst.sort()
    return out


def run_sharded(n_jobs: int, costs: Sequence[float], run: Callable[[list[int]], Sequence[int]],
                rank: int, world: int, group=None) -> np.ndarray | None:
    """Run this rank's share through `run(indices) -> per-job results` and gather
    all results, in job order, on rank 0 (None on the other ranks).  With
    world == 1 no process group is needed."""
    shards = shard_jobs(costs, world)
    mine = shards[rank]
    res = np.asarray(run(mine), dtype=np.int64)
    if res.shape != (len(mine),):
        raise ValueError("run() must return one result per job of the shard")
    if world == 1:
        return res
    import torch.distributed as dist

    parts = [None] * world if rank == 0 else None
    dist.gather_object(res.tolist(), parts, dst=0, group=group)
    if rank != 0:
        return None
    out = np.full(n_jobs, -1, dtype=np.int64)
    for r in range(world):
        out[shards[r]] = parts[r]
    return out
