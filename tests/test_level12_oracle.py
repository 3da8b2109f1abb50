"""CPU tests of the level-1 / level-2 oracle (oracle/level12.py): each
restatement against an independent scalar computation on small cases, the
triangular solve against its defining identity T X = B."""
import numpy as np
import pytest

import oracle as O
from oracle import level12 as L12

PRIMES = [2, 251, 65521, 2147483629, 4294967291]


def _rand(rng, p, shape):
    return rng.integers(0, p, shape, dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("p", PRIMES)
def test_gemv_axpy_scal_against_scalar_loops(p):
    rng = np.random.default_rng(p % 97)
    A, x, y = _rand(rng, p, (7, 9)), _rand(rng, p, 9), _rand(rng, p, 7)
    for op in (0, 1, 2):
        got = L12.gemv(p, A, x, y, op)
        for i in range(7):
            d = sum(int(A[i, t]) * int(x[t]) for t in range(9)) % p
            want = d if op == 0 else (int(y[i]) + d) % p if op == 1 else (int(y[i]) - d) % p
            assert int(got[i]) == want
    a = int(rng.integers(0, p))
    X, Y = _rand(rng, p, (4, 5)), _rand(rng, p, (4, 5))
    for sub in (False, True):
        got = L12.axpy(p, a, X, Y, sub)
        want = [[(int(Y[i, j]) + (-1 if sub else 1) * a * int(X[i, j])) % p for j in range(5)] for i in range(4)]
        assert got.tolist() == want
    assert L12.scal(p, a, X).tolist() == [[a * int(v) % p for v in r] for r in X]


@pytest.mark.parametrize("p", [251, 4294967291])
def test_gather_identity_and_row_lists(p):
    rng = np.random.default_rng(5)
    a = _rand(rng, p, (6, 8))
    c = _rand(rng, p, (3, 4))
    rows = np.array([5, 0, 3], np.uint32)
    cols = np.array([7, 3, 0, 5], np.uint32)
    alpha, beta, off = 3 % p, 11 % p, 2
    for acc in (False, True):
        got = L12.gather(p, alpha, beta, a, off, cols, c, acc, rows)
        for i in range(3):
            for t in range(4):
                v = (beta * int(a[rows[i], cols[t]]) + (alpha if off + rows[i] == cols[t] else 0)) % p
                want = (int(c[i, t]) + v) % p if acc else v
                assert int(got[i, t]) == want
    # identity source only, no index lists
    got = L12.gather(p, alpha, 0, None, 1, None, np.zeros((3, 4), np.uint32), False)
    want = np.zeros((3, 4), np.uint32)
    for i in range(3):
        want[i, i + 1] = alpha
    assert np.array_equal(got, want)


def test_canonicalise_forms():
    p = 2147483629
    v = np.array([[0, p - 1, p, 2 * p - 1]], np.uint32)
    assert L12.canonicalise(p, v).tolist() == [[0, p - 1, 0, p - 1]]
    acc = np.array([[0, 2**64 - 1, p * 12345 + 7]], np.uint64)
    assert L12.canonicalise_acc64(p, acc).tolist() == [[0, (2**64 - 1) % p, 7]]


@pytest.mark.parametrize("p", PRIMES)
@pytest.mark.parametrize("lower", [True, False])
def test_trsm_unit_solves_the_system(p, lower):
    rng = np.random.default_rng(3 + lower)
    m, n = 37, 5
    T = _rand(rng, p, (m, m))
    B = _rand(rng, p, (m, n))
    X = L12.trsm_unit(p, T, B, lower)
    Tu = (np.tril(T, -1) if lower else np.triu(T, 1)) + np.eye(m, dtype=np.uint32)
    assert np.array_equal(O.gemm(p, Tu, X), B)


def test_axpy_identity_on_a_wide_window():
    p = 65521
    y = np.full((3, 5), 65520, np.uint32)
    got = L12.axpy_identity(p, 2, y, False)
    assert [int(got[i, i]) for i in range(3)] == [1, 1, 1] and int(got[0, 1]) == 65520
