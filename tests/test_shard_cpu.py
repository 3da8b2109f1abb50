"""Multi-rank job stream on CPU: the deterministic cost-balanced assignment and
the host-side gather, run as two gloo ranks.  The per-job work is the oracle's
GEMM + rank of a small stream, so the gathered ranks are checked against a
single-process run of the same jobs."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from hacs_b200 import gen
from hacs_b200.shard import job_cost, run_sharded, shard_jobs

N_JOBS = 24


def _stream():
    s, fam, p, sa, sb = gen.job_stream(N_JOBS, salt=0x51)
    s = np.minimum(s, 48)  # small sides: the oracle runs the jobs in well under a second
    return s, fam, p, sa, sb


def _run_jobs(idx):
    import oracle

    s, fam, p, sa, sb = _stream()
    out = []
    for j in idx:
        n = int(s[j])
        A = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sa[j]))
        B = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sb[j]))
        C = oracle.gemm(int(p[j]), A, B)
        _, piv = oracle.rref(int(p[j]), C)
        out.append(len(piv))
    return out


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = _stream()[0]
        res = run_sharded(N_JOBS, job_cost(s, s, s), _run_jobs, rank, world)
        if rank == 0:
            q.put(res.tolist())
    finally:
        dist.destroy_process_group()


def test_shard_assignment_partitions_and_balances():
    costs = job_cost(*(np.arange(1, 41),) * 3)
    for world in (1, 2, 3, 8):
        sh = shard_jobs(costs, world)
        flat = sorted(j for lst in sh for j in lst)
        assert flat == list(range(40))
        assert all(lst == sorted(lst) for lst in sh)
        loads = [costs[lst].sum() for lst in sh]
        # LPT bound: the heaviest rank carries at most the mean plus the largest job
        assert max(loads) <= costs.sum() / world + costs.max()
    assert shard_jobs(costs, 2) == shard_jobs(costs.copy(), 2)  # deterministic
    with pytest.raises(ValueError):
        shard_jobs(costs, 0)


def test_two_gloo_ranks_gather_equals_single_run():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    try:
        got = q.get(timeout=120)
    finally:
        for pr in procs:
            pr.join(timeout=60)
    assert all(pr.exitcode == 0 for pr in procs)
    want = _run_jobs(list(range(N_JOBS)))
    assert got == want


def test_row_blocks_cover_and_align():
    from hacs_b200.shard import row_blocks

    for m in (1, 127, 128, 1000, 8192, 8200):
        for world in (1, 2, 3, 8):
            b = row_blocks(m, world)
            assert b[0][0] == 0 and b[-1][1] == m
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            assert all(r0 % 128 == 0 or r0 == m for r0, _ in b)
            sizes = [-(-(r1 - r0) // 128) for r0, r1 in b]
            assert max(sizes) - min(sizes) <= 1


def _gemm_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch

    import oracle
    from hacs_b200.shard import gemm_row_split

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        p = 2147483629
        A = torch.from_numpy(gen.engine_matrix(300, 70, p, 0x01).view(np.int32))
        B = torch.from_numpy(gen.engine_matrix(70, 90, p, 0x02).view(np.int32))

        def block_gemm(pp, Ab, Bb):  # each rank's own product of its row block (the oracle stands in for a GPU)
            Cb = oracle.gemm(pp, Ab.numpy().view(np.uint32), Bb.numpy().view(np.uint32))
            return torch.from_numpy(Cb.view(np.int32))

        C = gemm_row_split(block_gemm, p, A, B, rank, world)
        q.put((rank, C.numpy().view(np.uint32).tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_row_split_gemm_equals_single_product():
    """A 300-row product split over two ranks (blocks of 128-row tiles: 256 + 44
    rows), all-gathered: every rank holds the whole C, equal to one product."""
    import oracle

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gemm_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    try:
        got = dict(q.get(timeout=120) for _ in range(2))
    finally:
        for pr in procs:
            pr.join(timeout=60)
    assert all(pr.exitcode == 0 for pr in procs)
    p = 2147483629
    want = oracle.gemm(p, gen.engine_matrix(300, 70, p, 0x01), gen.engine_matrix(70, 90, p, 0x02))
    for r in range(2):
        assert np.array_equal(np.array(got[r], dtype=np.uint32), want)
