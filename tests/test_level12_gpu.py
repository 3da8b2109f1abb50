"""The device level-1 / level-2 entry points (through the C ABI) bit-exact
against the oracle: strided and transposed windows, every op, all limb
counts, empty shapes, index-list gathers, triangular solves across block
boundaries, and the contract checks of the reference (alpha canonical,
overlapping windows refused)."""
import numpy as np
import pytest

import hacs_b200
from oracle import level12 as L12

pytestmark = pytest.mark.gpu

PRIMES = [2, 251, 65521, 16777213, 2147483629, 4294967291]


def _rand(rng, p, shape):
    return rng.integers(0, p, shape, dtype=np.uint64).astype(np.uint32)


def _dev(M):
    import torch

    return torch.from_numpy(np.ascontiguousarray(M).view(np.int32)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint32)


def _windowed(rng, p, rows, cols, transposed):
    """A rows x cols window inside a larger random buffer (row stride > cols),
    or the transpose of such a window (row stride 1), and the buffer."""
    big = _dev(_rand(rng, p, (cols + 7, rows + 5) if transposed else (rows + 5, cols + 7)))
    return (big[3 : 3 + cols, 2 : 2 + rows].t() if transposed else big[3 : 3 + rows, 2 : 2 + cols]), big


@pytest.mark.parametrize("p", PRIMES)
@pytest.mark.parametrize("transposed", [False, True])
def test_gemv_all_ops_and_layouts(engine, p, transposed):
    rng = np.random.default_rng(p % 1009 + transposed)
    for m, k in [(1, 1), (33, 700), (300, 45), (129, 4096)]:
        A, _ = _windowed(rng, p, m, k, transposed)
        xs = _dev(_rand(rng, p, (k, 3)))
        x = xs[:, 1]  # a strided column
        for op in (hacs_b200.SET, hacs_b200.ADD, hacs_b200.SUB):
            y0 = _rand(rng, p, m)
            y = _dev(y0.reshape(1, m))[0]
            engine.gemv_dev(p, A, x, y, op)
            engine.sync()
            want = L12.gemv(p, _host(A.contiguous()), _host(x.contiguous()), y0, op)
            assert np.array_equal(_host(y), want), (m, k, op)


@pytest.mark.parametrize("p", PRIMES)
def test_elementwise_ops_on_strided_windows(engine, p):
    rng = np.random.default_rng(p % 4001)
    for rows, cols in [(1, 1), (17, 300), (640, 3), (70, 2100)]:
        for tr in (False, True):
            alpha = int(rng.integers(0, p))
            x, _ = _windowed(rng, p, rows, cols, tr)
            y, ybig = _windowed(rng, p, rows, cols, not tr)
            yb0 = _host(ybig).copy()
            for sub in (False, True):
                xh, yh = _host(x.contiguous()), _host(y.contiguous())
                engine.axpy_dev(p, alpha, x, y, sub)
                engine.sync()
                assert np.array_equal(_host(y.contiguous()), L12.axpy(p, alpha, xh, yh, sub))
            # cells of the buffer outside the window are untouched
            yb1 = _host(ybig)
            mask = np.ones_like(yb1, bool)
            if not tr:  # y is a transposed window: buffer rows 3.., columns 2..
                mask[3 : 3 + cols, 2 : 2 + rows] = False
            else:
                mask[3 : 3 + rows, 2 : 2 + cols] = False
            assert np.array_equal(yb1[mask], yb0[mask])
            xh = _host(x.contiguous())
            engine.scal_dev(p, alpha, x)
            engine.sync()
            assert np.array_equal(_host(x.contiguous()), L12.scal(p, alpha, xh))
            engine.copy_dev(x, y)
            engine.sync()
            assert np.array_equal(_host(y.contiguous()), _host(x.contiguous()))
            engine.fill_dev(y, 12345 % p)
            engine.sync()
            assert (_host(y.contiguous()) == 12345 % p).all()


@pytest.mark.parametrize("shape", [(1, 1), (31, 33), (64, 64), (1000, 37), (5, 4097)])
def test_transpose(engine, shape):
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    r, c = shape
    src, _ = _windowed(rng, 2**32 - 5, r, c, False)
    dst, _ = _windowed(rng, 2**32 - 5, c, r, False)
    engine.transpose_dev(src, dst)
    engine.sync()
    assert np.array_equal(_host(dst.contiguous()), _host(src.contiguous()).T)
    dst2, _ = _windowed(rng, 2**32 - 5, c, r, True)
    engine.transpose_dev(src, dst2)
    engine.sync()
    assert np.array_equal(_host(dst2.contiguous()), _host(src.contiguous()).T)


@pytest.mark.parametrize("p", [251, 2147483629])
def test_axpy_identity_and_canonicalise(engine, p):
    rng = np.random.default_rng(9)
    for rows, cols in [(5, 9), (9, 5), (300, 300)]:
        y, _ = _windowed(rng, p, rows, cols, False)
        y0 = _host(y.contiguous())
        a = int(rng.integers(0, p))
        for sub in (False, True):
            engine.axpy_identity_dev(p, a, y, sub)
            engine.sync()
            y0 = L12.axpy_identity(p, a, y0, sub)
            assert np.array_equal(_host(y.contiguous()), y0)
    lazy = rng.integers(0, 2 * p, (70, 90), dtype=np.uint64).astype(np.uint32)
    v = _dev(lazy)
    engine.canonicalise_dev(p, v[:, 10:80])
    engine.sync()
    want = lazy.copy()
    want[:, 10:80] = L12.canonicalise(p, lazy[:, 10:80])
    assert np.array_equal(_host(v), want)


@pytest.mark.parametrize("p", [65521, 2147483629, 4294967291])
def test_canonicalise_acc64(engine, p):
    import torch

    rng = np.random.default_rng(p % 13)
    acc = rng.integers(0, 2**64 - 1, (129, 65), dtype=np.uint64, endpoint=True)
    acc[0, 0], acc[0, 1] = 0, 2**64 - 1
    a = torch.from_numpy(acc.view(np.int64)).cuda()
    d = torch.zeros((65, 129), dtype=torch.int32, device="cuda")
    engine.canonicalise_acc64_dev(p, a, d.t())
    engine.sync()
    assert np.array_equal(_host(d).T, L12.canonicalise_acc64(p, acc))


@pytest.mark.parametrize("p", [251, 4294967291])
def test_gather_forms(engine, p):
    import torch

    rng = np.random.default_rng(21)
    a_h = _rand(rng, p, (200, 1500))
    a = _dev(a_h)
    rows_h = rng.integers(0, 200, 70).astype(np.uint32)
    cols_h = rng.integers(0, 1500, 1100).astype(np.uint32)
    rows = torch.from_numpy(rows_h.view(np.int32)).cuda()
    cols = torch.from_numpy(cols_h.view(np.int32)).cuda()
    alpha, beta = int(rng.integers(0, p)), int(rng.integers(1, p))
    for acc in (False, True):
        for r_l, c_l, shape in [(None, None, (200, 1500)), (rows, None, (70, 1500)), (None, cols, (200, 1100)),
                                (rows, cols, (70, 1100))]:
            c0 = _rand(rng, p, shape)
            c = _dev(c0)
            engine.gather_dev(p, alpha, beta, a, 17, c_l, c, acc, r_l)
            engine.sync()
            want = L12.gather(p, alpha, beta, a_h, 17, None if c_l is None else cols_h, c0, acc,
                              None if r_l is None else rows_h)
            assert np.array_equal(_host(c), want)
    c0 = _rand(rng, p, (40, 50))
    c = _dev(c0)
    engine.gather_dev(p, alpha, 0, None, 3, None, c, True)
    engine.sync()
    assert np.array_equal(_host(c), L12.gather(p, alpha, 0, None, 3, None, c0, True))


@pytest.mark.parametrize("p", PRIMES)
@pytest.mark.parametrize("lower", [True, False])
def test_trsm_unit(engine, p, lower):
    rng = np.random.default_rng(p % 311 + lower)
    for m, n in [(1, 3), (31, 7), (32, 32), (33, 300), (129, 65), (300, 1), (400, 70)]:
        T_h = _rand(rng, p, (m, m + 3))
        B_h = _rand(rng, p, (m, n + 5))
        T, B = _dev(T_h), _dev(B_h)
        engine.trsm_unit_dev(p, T[:, :m], B[:, :n], lower)
        engine.sync()
        want = B_h.copy()
        want[:, :n] = L12.trsm_unit(p, T_h[:, :m], B_h[:, :n], lower)
        assert np.array_equal(_host(B), want), (m, n)


@pytest.mark.parametrize("p", PRIMES)
def test_gemm_nt_and_schur_update(engine, p):
    import torch

    rng = np.random.default_rng(p % 577)
    for m, n, k in [(1, 1, 1), (64, 200, 3), (300, 129, 500), (128, 128, 0)]:
        A_h, B_h = _rand(rng, p, (m, k)), _rand(rng, p, (n, k))
        for op in (hacs_b200.SET, hacs_b200.ADD, hacs_b200.SUB):
            C_h = _rand(rng, p, (m, n))
            C = _dev(C_h)
            A = _dev(A_h) if k else torch.zeros((m, 0), dtype=torch.int32, device="cuda")
            B = _dev(B_h) if k else torch.zeros((n, 0), dtype=torch.int32, device="cuda")
            engine.gemm_nt_dev(p, A, B, C, op)
            engine.sync()
            assert np.array_equal(_host(C), L12.gemm_nt(p, A_h, B_h, C_h, op)), (m, n, k, op)
        if k:
            C_h = _rand(rng, p, (m, n))
            C = _dev(C_h)
            engine.schur_update_dev(p, _dev(A_h), _dev(np.ascontiguousarray(B_h.T)), C)
            engine.sync()
            assert np.array_equal(_host(C), L12.gemm_nt(p, A_h, B_h, C_h, hacs_b200.SUB))


def test_contract_checks(engine):
    import torch

    p = 65521
    x = torch.zeros((10, 10), dtype=torch.int32, device="cuda")
    with pytest.raises(hacs_b200.HmeError):
        engine.axpy_dev(p, p, x, x.clone())  # alpha not canonical
    with pytest.raises(hacs_b200.HmeError):
        engine.copy_dev(x[0:5], x[3:8])  # overlapping windows
    with pytest.raises(hacs_b200.HmeError):
        engine.trsm_unit_dev(p, x, x, True)  # T aliases B
    with pytest.raises(hacs_b200.HmeError):
        engine.gather_dev(p, 1, 1, x, 0, None, x[2:4], False)  # row count mismatch, output aliases the source
    y = torch.zeros((0, 5), dtype=torch.int32, device="cuda")
    engine.fill_dev(y, 3)  # empty views are no-ops
    engine.copy_dev(x, x)  # a self-copy is a no-op
    engine.sync()


@pytest.mark.parametrize("p", [251, 65521, 2147483629, 4294967291])
def test_vector_paths_on_aligned_views(engine, p):
    """16-byte vector paths: contiguous operands and windows whose rows start
    16-byte aligned (column offset 4, row stride a multiple of 4), next to a
    window one column off alignment (scalar path) in the same buffer."""
    import torch

    rng = np.random.default_rng(p % 7919)
    for rows, cols in [(1, 4), (3, 1024), (257, 4100), (4096, 64)]:
        for c0 in (4, 5):
            xb = _dev(_rand(rng, p, (rows, cols + 12)))
            yb0 = _rand(rng, p, (rows, cols + 12))
            yb = _dev(yb0)
            x, y = xb[:, c0 : c0 + cols], yb[:, c0 : c0 + cols]
            alpha = int(rng.integers(0, p))
            xh, yh = _host(x.contiguous()), _host(y.contiguous())
            engine.axpy_dev(p, alpha, x, y, True)
            engine.sync()
            assert np.array_equal(_host(y.contiguous()), L12.axpy(p, alpha, xh, yh, True)), (rows, cols, c0)
            engine.scal_dev(p, alpha, y)
            engine.sync()
            yh = L12.axpy(p, alpha, xh, yh, True)
            assert np.array_equal(_host(y.contiguous()), L12.scal(p, alpha, yh))
            engine.copy_dev(x, y)
            engine.fill_dev(x, 7 % p)
            engine.sync()
            assert np.array_equal(_host(y.contiguous()), xh)
            assert (_host(x.contiguous()) == 7 % p).all()
            # the buffer's columns outside the window are untouched
            out = _host(yb)
            assert np.array_equal(out[:, :c0], yb0[:, :c0]) and np.array_equal(out[:, c0 + cols :], yb0[:, c0 + cols :])
    if p <= 2**31:
        lazy = rng.integers(0, 2 * p, (300, 516), dtype=np.uint64).astype(np.uint32)
        v = _dev(lazy)
        engine.canonicalise_dev(p, v[:, 4:516])
        engine.sync()
        want = lazy.copy()
        want[:, 4:516] = L12.canonicalise(p, lazy[:, 4:516])
        assert np.array_equal(_host(v), want)
    acc = rng.integers(0, 2**64 - 1, (100, 1028), dtype=np.uint64, endpoint=True)
    a = torch.from_numpy(acc.view(np.int64)).cuda()
    d = torch.zeros((100, 1028), dtype=torch.int32, device="cuda")
    engine.canonicalise_acc64_dev(p, a, d)
    engine.sync()
    assert np.array_equal(_host(d), L12.canonicalise_acc64(p, acc))
    for m, k in [(1, 4), (65, 8192), (1000, 516), (3, 50000), (2, 50001)]:  # the last two: x not staged
        A_h, x_h, y0 = _rand(rng, p, (m, k)), _rand(rng, p, k), _rand(rng, p, m)
        y = _dev(y0.reshape(1, m))[0]
        engine.gemv_dev(p, _dev(A_h), _dev(x_h.reshape(1, k))[0], y, hacs_b200.ADD)
        engine.sync()
        assert np.array_equal(_host(y), L12.gemv(p, A_h, x_h, y0, hacs_b200.ADD)), (m, k)


@pytest.mark.parametrize("p", [251, 4294967291])
def test_gather_identity_vector_path(engine, p):
    """The 4-column gather with no source (identity term only) and with a
    source and row list, windows aligned for 16-byte accesses."""
    import torch

    rng = np.random.default_rng(p % 101)
    for acc in (False, True):
        c0 = _rand(rng, p, (64, 128))
        c = _dev(c0)
        engine.gather_dev(p, 5 % p, 0, None, 3, None, c, acc)
        engine.sync()
        assert np.array_equal(_host(c), L12.gather(p, 5 % p, 0, None, 3, None, c0, acc))
    a_h = _rand(rng, p, (90, 256))
    rows_h = rng.permutation(90)[:40].astype(np.uint32)
    c0 = _rand(rng, p, (40, 256))
    c = _dev(c0)
    engine.gather_dev(p, 9 % p, 7 % p, _dev(a_h), 1, None, c, True, torch.from_numpy(rows_h.view(np.int32)).cuda())
    engine.sync()
    assert np.array_equal(_host(c), L12.gather(p, 9 % p, 7 % p, a_h, 1, None, c0, True, rows_h))


def test_device_ops_reproduce_reference_golden_vectors(engine):
    """The device entry points reproduce the reference CPU engine's FNV
    checksums: the micro bench's gemv (salts 3 / 4) and transpose (salt 5)
    workloads, A*B^T, axpy / scal, both canonicalisations and the triangular
    solves (fixtures in tests/golden/level12.json)."""
    import json
    import os

    import torch

    from hacs_b200 import gen

    G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "level12.json")))

    def fnv(t):
        import oracle as O

        return "0x%016x" % O.fnv_matrix(np.ascontiguousarray(_host(t)))

    for g in G["micro_gemv"]:
        n, p = g["n"], g["p"]
        y = torch.zeros((n, 1), dtype=torch.int32, device="cuda")
        engine.gemv_dev(p, _dev(gen.engine_matrix(n, n, p, 3)), _dev(gen.engine_matrix(n, 1, p, 4)), y)
        engine.sync()
        assert fnv(y) == g["fnv"], g
    for g in G["micro_transpose"]:
        n = g["n"]
        T = torch.zeros((n, n), dtype=torch.int32, device="cuda")
        engine.transpose_dev(_dev(gen.engine_matrix(n, n, g["p"], 5)), T)
        engine.sync()
        assert fnv(T) == g["fnv"], g
    for g in G["gemm_nt"]:
        m, n, k, p = g["m"], g["n"], g["k"], g["p"]
        C = _dev(gen.engine_matrix(m, n, p, 8))
        engine.gemm_nt_dev(p, _dev(gen.engine_matrix(m, k, p, 6)), _dev(gen.engine_matrix(n, k, p, 7)), C, g["op"])
        engine.sync()
        assert fnv(C) == g["fnv"], g
    for g in G["axpy_scal"]:
        r, c, p, a = g["rows"], g["cols"], g["p"], g["alpha"]
        for sub, key in ((False, "axpy_fnv"), (True, "axpy_sub_fnv")):
            y = _dev(gen.engine_matrix(r, c, p, 10))
            engine.axpy_dev(p, a, _dev(gen.engine_matrix(r, c, p, 9)), y, sub)
            engine.sync()
            assert fnv(y) == g[key], g
        x = _dev(gen.engine_matrix(r, c, p, 9))
        engine.scal_dev(p, a, x)
        engine.sync()
        assert fnv(x) == g["scal_fnv"], g
    for g in G["canonicalise"]:
        r, c, p = g["rows"], g["cols"], g["p"]
        v = _dev(gen.engine_matrix(r, c, 2 * p, 11))
        engine.canonicalise_dev(p, v)
        hi = gen.engine_matrix(r, c, 4294967291, 12).astype(np.uint64)
        lo = gen.engine_matrix(r, c, 4294967291, 13).astype(np.uint64)
        acc = torch.from_numpy(((hi << np.uint64(32)) | lo).view(np.int64)).cuda()
        d = torch.zeros((r, c), dtype=torch.int32, device="cuda")
        engine.canonicalise_acc64_dev(p, acc, d)
        engine.sync()
        assert fnv(v) == g["lazy_fnv"] and fnv(d) == g["acc64_fnv"], g
    for g in G["trsm"]:
        m, n, p = g["m"], g["n"], g["p"]
        B = _dev(gen.engine_matrix(m, n, p, 15))
        engine.trsm_unit_dev(p, _dev(gen.engine_matrix(m, m, p, 14)), B, g["lower"])
        engine.sync()
        assert fnv(B) == g["fnv"], g
