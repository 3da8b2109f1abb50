"""Parity of the INT8-limb tcgen05 GEMM (through the C ABI) with the oracle.

Bit-exact comparison: every output residue must equal the oracle's
(oracle/oracle.c orc_gemm_u32, pinned to the reference's
engine::kernels::gemm<uint32_t>)."""
import numpy as np
import pytest

import oracle as O
from hacs_b200 import ADD, SET, SUB
from hacs_b200 import gen

pytestmark = pytest.mark.gpu

PRIMES = [2, 3, 13, 251, 257, 65521, 65536, 16777213, 16777259, 134217757, 2147483629, 2147483647, 4294967291]


def _rand(rng, shape, p):
    return rng.integers(0, p, shape, dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("p", PRIMES)
def test_gemm_square_all_ops(engine, p):
    rng = np.random.default_rng(p % 1000)
    for (m, n, k) in [(1, 1, 1), (128, 128, 128), (200, 72, 300)]:
        A, B, C0 = _rand(rng, (m, k), p), _rand(rng, (k, n), p), _rand(rng, (m, n), p)
        for op in (SET, ADD, SUB):
            got = engine.gemm(p, A, B, C0, op)
            want = O.gemm(p, A, B, C0, op)
            assert np.array_equal(got, want), (p, m, n, k, op)


@pytest.mark.parametrize("m,n,k", [(1, 300, 17), (129, 1, 5), (17, 33, 1000), (300, 257, 129), (513, 130, 2049)])
@pytest.mark.parametrize("p", [65521, 2147483629])
def test_gemm_ragged_shapes(engine, p, m, n, k):
    rng = np.random.default_rng(m * 7 + n)
    A, B = _rand(rng, (m, k), p), _rand(rng, (k, n), p)
    assert np.array_equal(engine.gemm(p, A, B), O.gemm(p, A, B))


@pytest.mark.parametrize("p", [65521, 2147483629, 4294967291])
def test_gemm_worst_case_all_pminus1(engine, p):
    # every entry p-1 over several K chunks: the largest limb sums the accumulator sees
    m, n = 130, 140
    k = 9000 if p > 65536 else 17000
    A = np.full((m, k), p - 1, np.uint32)
    B = np.full((k, n), p - 1, np.uint32)
    got = engine.gemm(p, A, B)
    want = (k % p) * ((p - 1) * (p - 1) % p) % p
    assert np.all(got == want)


def test_gemm_config1_checksum(engine):
    """Config 1: 1024^3, p = 65521, EngineMatrix salts 0x01 / 0x02 -- the
    reference's `--bench micro gemm 1024 1024 65521` inputs; bit-exact."""
    p, n = 65521, 1024
    A = gen.engine_matrix(n, n, p, 0x01)
    B = gen.engine_matrix(n, n, p, 0x02)
    got = engine.gemm(p, A, B)
    want = O.gemm(p, A, B)
    assert np.array_equal(got, want)
    assert gen.fnv_matrix(got) == 0x572E8347446366C6


@pytest.mark.parametrize("p", [251, 65521, 16777213, 2147483629])
def test_gemm_wide_tiles(engine, p):
    # enough output tiles that the wide-tile variant (L*BN = 256) is chosen
    rng = np.random.default_rng(p % 97)
    m, n, k = 2048, 2304, 160
    A, B, C0 = _rand(rng, (m, k), p), _rand(rng, (k, n), p), _rand(rng, (m, n), p)
    assert np.array_equal(engine.gemm(p, A, B, C0, SUB), O.gemm(p, A, B, C0, SUB))


def test_gemm_device_pointers_strided(engine):
    """hme_gemm_u32_dev on torch CUDA tensors with padded leading dimensions."""
    import torch

    p = 2147483629
    rng = np.random.default_rng(3)
    m, n, k = 300, 200, 500
    A, B, C0 = _rand(rng, (m, k), p), _rand(rng, (k, n), p), _rand(rng, (m, n), p)
    dA = torch.zeros((m, k + 7), dtype=torch.int32, device="cuda")
    dB = torch.zeros((k, n + 3), dtype=torch.int32, device="cuda")
    dC = torch.zeros((m, n + 5), dtype=torch.int32, device="cuda")
    dA[:, :k] = torch.from_numpy(A.view(np.int32))
    dB[:, :n] = torch.from_numpy(B.view(np.int32))
    dC[:, :n] = torch.from_numpy(C0.view(np.int32))
    engine.use_torch_stream()
    engine.gemm_dev(p, dA[:, :k], dB[:, :n], dC[:, :n], ADD)
    engine.sync()
    got = dC[:, :n].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, O.gemm(p, A, B, C0, ADD))
    assert np.all(dC[:, n:].cpu().numpy() == 0)  # padding untouched


@pytest.mark.parametrize("p,m,n,k,op", [
    (65521, 2000, 1100, 300, SET),      # 4 row chunks (>= 2 MiB of C each), the last one ragged
    (2147483629, 1500, 1500, 200, SUB), # 4 limbs, Sub: C's rows are copied in chunk by chunk
    (65521, 1000, 300, 700, SET),       # one chunk
    (251, 640, 1024, 129, ADD),         # 1 limb
    (16777213, 129, 64, 12000, SET),    # 3 limbs, K beyond one exact-accumulation chunk, 2 row chunks
])
def test_gemm_host_pointers_strided_pipeline(engine, p, m, n, k, op):
    """hme_gemm_u32 (host pointers) with leading dimensions larger than the
    rows: the chunked copy/compute pipeline must read and write only the
    m x n (m x k, k x n) windows."""
    import ctypes as C

    from hacs_b200 import check

    rng = np.random.default_rng(m + n + k)
    lda, ldb, ldc = k + 5, n + 3, n + 9
    Ah = _rand(rng, (m, lda), p)
    Bh = _rand(rng, (k, ldb), p)
    Ch = _rand(rng, (m, ldc), p)
    want = O.gemm(p, Ah[:, :k], Bh[:, :n], Ch[:, :n].copy(), op)
    pad = Ch[:, n:].copy()
    u = C.POINTER(C.c_uint32)
    rc = engine._lib.hme_gemm_u32(engine._h, p, m, n, k, Ah.ctypes.data_as(u), lda, Bh.ctypes.data_as(u), ldb,
                                  Ch.ctypes.data_as(u), ldc, op)
    check(rc)
    assert np.array_equal(Ch[:, :n], want)
    assert np.array_equal(Ch[:, n:], pad)


def test_gemm_and_rref_on_every_visible_device():
    """Kernel attributes (the large dynamic shared memory of the limb GEMM, the
    elimination's cluster and block kernels) are set once per device, not once
    per process: a context on each visible device runs a GEMM and an RREF in the
    same process, bit-exact (skipped with a single visible device)."""
    import torch

    import hacs_b200

    n_dev = torch.cuda.device_count()
    if n_dev < 2:
        pytest.skip("one visible device")
    rng = np.random.default_rng(77)
    p = 2147483629
    A, B = _rand(rng, (300, 257), p), _rand(rng, (257, 190), p)
    want = O.gemm(p, A, B)
    M = _rand(rng, (150, 140), p)
    want_r, want_p = O.rref(p, M)
    engines = [hacs_b200.Engine(d) for d in range(n_dev)]
    try:
        for e in engines + engines[::-1]:
            assert np.array_equal(e.gemm(p, A, B), want)
            R, piv = e.rref(p, M)
            assert np.array_equal(R, want_r) and np.array_equal(piv, want_p)
    finally:
        for e in engines:
            e.close()
