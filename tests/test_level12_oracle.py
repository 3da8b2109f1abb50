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


# ---- pinned against the reference's own CPU kernels ----------------------------
import json  # noqa: E402
import os  # noqa: E402

from hacs_b200 import gen  # noqa: E402

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "level12.json")))


def _fnv(M):
    return "0x%016x" % O.fnv_matrix(np.ascontiguousarray(M, dtype=np.uint32))


def _acc64(rows, cols, p, salt_hi, salt_lo):
    hi = gen.engine_matrix(rows, cols, p, salt_hi).astype(np.uint64)
    lo = gen.engine_matrix(rows, cols, 4294967291, salt_lo).astype(np.uint64)
    return (hi << np.uint64(32)) | lo


def test_oracle_reproduces_reference_golden_vectors():
    """Every level-1 / level-2 fixture (FNV of the reference CPU engine's
    output on EngineMatrix inputs) is reproduced by the restatement."""
    for g in GOLD["micro_gemv"]:
        n, p = g["n"], g["p"]
        A, x = gen.engine_matrix(n, n, p, 3), gen.engine_matrix(n, 1, p, 4)
        assert _fnv(L12.gemv(p, A, x, np.zeros(n, np.uint32), 0).reshape(n, 1)) == g["fnv"]
    for g in GOLD["micro_transpose"]:
        assert _fnv(gen.engine_matrix(g["n"], g["n"], g["p"], 5).T) == g["fnv"]
    for g in GOLD["gemm_nt"]:
        m, n, k, p = g["m"], g["n"], g["k"], g["p"]
        A, B, C = gen.engine_matrix(m, k, p, 6), gen.engine_matrix(n, k, p, 7), gen.engine_matrix(m, n, p, 8)
        assert _fnv(L12.gemm_nt(p, A, B, C, g["op"])) == g["fnv"]
    for g in GOLD["axpy_scal"]:
        r, c, p, a = g["rows"], g["cols"], g["p"], g["alpha"]
        x, y = gen.engine_matrix(r, c, p, 9), gen.engine_matrix(r, c, p, 10)
        assert _fnv(L12.axpy(p, a, x, y, False)) == g["axpy_fnv"]
        assert _fnv(L12.axpy(p, a, x, y, True)) == g["axpy_sub_fnv"]
        assert _fnv(L12.scal(p, a, x)) == g["scal_fnv"]
    for g in GOLD["canonicalise"]:
        r, c, p = g["rows"], g["cols"], g["p"]
        assert _fnv(L12.canonicalise(p, gen.engine_matrix(r, c, 2 * p, 11))) == g["lazy_fnv"]
        assert _fnv(L12.canonicalise_acc64(p, _acc64(r, c, 4294967291, 12, 13))) == g["acc64_fnv"]
    for g in GOLD["trsm"]:
        m, n, p = g["m"], g["n"], g["p"]
        T, B = gen.engine_matrix(m, m, p, 14), gen.engine_matrix(m, n, p, 15)
        assert _fnv(L12.trsm_unit(p, T, B, g["lower"])) == g["fnv"]


@pytest.mark.skipif(not O.ref_available(), reason="reference CPU engine not built here")
@pytest.mark.parametrize("p", [2, 251, 65521, 2147483629, 4294967291])
def test_oracle_matches_reference_kernels_directly(p):
    rng = np.random.default_rng(p % 1000 + 3)
    A, x, y = _rand(rng, p, (37, 61)), _rand(rng, p, 61), _rand(rng, p, 37)
    for op in (0, 1, 2):
        assert np.array_equal(L12.gemv(p, A, x, y, op), O.ref_gemv(p, A, x, y, op))
    B, C = _rand(rng, p, (29, 61)), _rand(rng, p, (37, 29))
    for op in (0, 1, 2):
        assert np.array_equal(L12.gemm_nt(p, A, B, C, op), O.ref_gemm_nt(p, A, B, C, op))
    a = int(rng.integers(0, p))
    X, Y = _rand(rng, p, (9, 33)), _rand(rng, p, (9, 33))
    for sub in (False, True):
        assert np.array_equal(L12.axpy(p, a, X, Y, sub), O.ref_axpy(p, a, X, Y, sub))
    assert np.array_equal(L12.scal(p, a, X), O.ref_scal(p, a, X))
    T, Bm = _rand(rng, p, (70, 70)), _rand(rng, p, (70, 11))
    for lower in (True, False):
        assert np.array_equal(O.ref_trmm_unit(p, T, L12.trsm_unit(p, T, Bm, lower), lower), Bm)
    if 2 * p < 2**32:
        lazy = rng.integers(0, 2 * p, (8, 13), dtype=np.uint64).astype(np.uint32)
        assert np.array_equal(L12.canonicalise(p, lazy), O.ref_canonicalise(p, lazy))
    acc = rng.integers(0, 2**64 - 1, (8, 13), dtype=np.uint64, endpoint=True)
    assert np.array_equal(L12.canonicalise_acc64(p, acc), O.ref_canonicalise_acc64(p, acc))
