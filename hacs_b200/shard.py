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


# ---- one large GEMM split by rows of C ------------------------------------------------------
def row_blocks(m: int, world: int, align: int = 128) -> list[tuple[int, int]]:
    """Rank r's rows [r0, r1) of an m-row product: contiguous blocks in rank
    order whose boundaries fall on multiples of `align` (the limb GEMM's 128-row
    tile), block sizes differing by at most one tile.  Deterministic, so every
    rank computes the same split without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    tiles = -(-m // align)
    out, t0 = [], 0
    for r in range(world):
        t1 = t0 + tiles // world + (1 if r < tiles % world else 0)
        out.append((min(m, t0 * align), min(m, t1 * align)))
        t0 = t1
    return out


def gemm_row_split(gemm: Callable, p: int, A, B, rank: int, world: int, group=None, align: int = 128):
    """C = A B mod p with C's rows split over the ranks (A's row block local,
    B replicated, no reduction since every C row has one owner).  Rank r computes its block with gemm(p, A[r0:r1], B) on its own
    device, then the blocks are all-gathered (torch.distributed, NCCL for CUDA
    tensors, gloo for CPU ones) so every rank returns the whole C.  A and B are
    torch tensors on this rank's device; gemm returns the block as a tensor."""
    import torch

    blocks = row_blocks(int(A.shape[0]), world, align)
    r0, r1 = blocks[rank]
    n = int(B.shape[1])
    Cb = gemm(p, A[r0:r1], B) if r1 > r0 else torch.empty((0, n), dtype=A.dtype, device=A.device)
    if world == 1:
        return Cb
    import torch.distributed as dist

    mx = max(b1 - b0 for b0, b1 in blocks)
    pad = torch.zeros((mx, n), dtype=Cb.dtype, device=Cb.device)
    pad[: r1 - r0] = Cb
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([parts[r][: b1 - b0] for r, (b0, b1) in enumerate(blocks)], dim=0)
