"""The u64-residue level-1 device operations (hme_*_u64_dev) through the C ABI
against the oracle's exact-integer restatements (oracle/level12.py): strided
and transposed windows, moduli from 2 to 2^64 - 59, and the contract checks."""
import ctypes as C

import numpy as np
import pytest

import oracle.level12 as R
from hacs_b200 import _lib

pytestmark = pytest.mark.gpu

PRIMES = [2, 65521, 2147483629, 2**61 - 1, 2**64 - 59]


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _h(t):
    return t.cpu().numpy().view(np.uint64)


def _rand(rng, shape, p):
    return rng.integers(0, p, shape, dtype=np.uint64)


def _rc(rc):
    assert rc == 0, _lib.lib().hme_last_error().decode()


@pytest.mark.parametrize("p", PRIMES)
def test_axpy_scal_fill_canonicalise_u64(engine, p):
    import torch

    L = _lib.lib()
    rng = np.random.default_rng(p % 1000003)
    m, n = 37, 53
    X, Y = _rand(rng, (m, n), p), _rand(rng, (m, n), p)
    alpha = int(_rand(rng, (1,), p)[0])
    engine.use_own_stream()
    for sub in (0, 1):
        x, y = _t(X), _t(Y)
        _rc(L.hme_axpy_u64_dev(engine._h, p, alpha, m, n, x.data_ptr(), n, 1, y.data_ptr(), n, 1, sub))
        engine.sync()
        assert np.array_equal(_h(y), R.axpy64(p, alpha, X, Y, bool(sub)))
    # transposed windows: y^T (n x m) += alpha x^T
    x, y = _t(X), _t(Y)
    _rc(L.hme_axpy_u64_dev(engine._h, p, alpha, n, m, x.data_ptr(), 1, n, y.data_ptr(), 1, n, 0))
    engine.sync()
    assert np.array_equal(_h(y), R.axpy64(p, alpha, X, Y, False))
    y = _t(Y)
    _rc(L.hme_scal_u64_dev(engine._h, p, alpha, m, n, y.data_ptr(), n, 1))
    engine.sync()
    assert np.array_equal(_h(y), R.scal64(p, alpha, Y))
    y = _t(Y)
    _rc(L.hme_fill_u64_dev(engine._h, m, n - 3, y.data_ptr(), n, 1, alpha))
    engine.sync()
    want = Y.copy()
    want[:, : n - 3] = alpha
    assert np.array_equal(_h(y), want)
    if p <= 2**63:
        lazy = (Y + rng.integers(0, 2, (m, n), dtype=np.uint64) * np.uint64(p))
        v = _t(lazy)
        _rc(L.hme_canonicalise_u64_dev(engine._h, p, m, n, v.data_ptr(), n, 1))
        engine.sync()
        assert np.array_equal(_h(v), R.canonicalise64(p, lazy))
    bad = L.hme_axpy_u64_dev(engine._h, p, p, m, n, x.data_ptr(), n, 1, y.data_ptr(), n, 1, 0)
    assert bad == _lib.HME_EINVAL  # alpha must be canonical


@pytest.mark.parametrize("shape", [(1, 1), (31, 33), (64, 64), (100, 7), (257, 130)])
def test_copy_transpose_u64(engine, shape):
    import torch

    L = _lib.lib()
    rng = np.random.default_rng(shape[0] * 1000 + shape[1])
    m, n = shape
    S = rng.integers(0, 2**63, (m, n), dtype=np.uint64) * np.uint64(2) + np.uint64(1)
    s = _t(S)
    d = torch.zeros((m, n + 2), dtype=torch.int64, device="cuda")
    _rc(L.hme_copy_u64_dev(engine._h, m, n, s.data_ptr(), n, 1, d.data_ptr(), n + 2, 1))
    t = torch.zeros((n, m), dtype=torch.int64, device="cuda")
    _rc(L.hme_transpose_u64_dev(engine._h, n, m, s.data_ptr(), n, 1, t.data_ptr(), m, 1))
    engine.sync()
    assert np.array_equal(_h(d)[:, :n], S)
    assert np.array_equal(_h(t), S.T)
    assert L.hme_copy_u64_dev(engine._h, m, n, s.data_ptr(), n, 1, s.data_ptr(), n, 1) == _lib.HME_EINVAL


@pytest.mark.parametrize("p", [65521, 2**61 - 1, 2**64 - 59])
def test_gather_and_identity_axpy_u64(engine, p):
    import torch

    L = _lib.lib()
    rng = np.random.default_rng(7 + p % 97)
    A = _rand(rng, (40, 30), p)
    Cm = _rand(rng, (12, 9), p)
    cols = rng.integers(0, 30, 9).astype(np.uint32)
    rows = rng.integers(0, 40, 12).astype(np.uint32)
    alpha, beta = int(_rand(rng, (1,), p)[0]), int(_rand(rng, (1,), p)[0])
    a, dc, dr = _t(A), torch.from_numpy(cols.view(np.int32)).cuda(), torch.from_numpy(rows.view(np.int32)).cuda()
    for acc in (0, 1):
        for use_rows in (False, True):
            c = _t(Cm)
            _rc(L.hme_gather_u64_dev(engine._h, p, alpha, beta, a.data_ptr(), 40, 30, 30, 1, 3, dc.data_ptr(),
                                     dr.data_ptr() if use_rows else None, 12, 9, c.data_ptr(), 9, 1, acc))
            engine.sync()
            want = R.gather64(p, alpha, beta, A, 3, cols, Cm, bool(acc), rows if use_rows else None)
            assert np.array_equal(_h(c), want), (acc, use_rows)
    Y = _rand(rng, (9, 14), p)
    for sub in (0, 1):
        y = _t(Y)
        _rc(L.hme_axpy_identity_u64_dev(engine._h, p, alpha, 9, 14, y.data_ptr(), 14, 1, sub))
        engine.sync()
        assert np.array_equal(_h(y), R.axpy_identity64(p, alpha, Y, bool(sub)))
