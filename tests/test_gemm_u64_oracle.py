"""CPU tests of the u64-residue GEMM oracle (oracle.c orc_gemm_u64): against
exact Python integers, against the reference's kernels::gemm<uint64_t>
(where oracle/_ref is built) and against the committed golden checksums."""
import json
import os

import numpy as np
import pytest

import oracle as O

MODULI = [2, 134217757, 4294967311, 1099511627776, 10**12, 2305843009213693951, 9223372036854775783,
          9223372036854775837, 18446744073709551557]
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "level12.json")))


def _exact(p, A, B, C, op):
    m, k = A.shape
    n = B.shape[1]
    out = np.zeros((m, n), np.uint64)
    for i in range(m):
        for j in range(n):
            s = sum(int(A[i, t]) * int(B[t, j]) for t in range(k))
            old = int(C[i, j])
            out[i, j] = s % p if op == 0 else (old + s) % p if op == 1 else (old - s) % p
    return out


@pytest.mark.parametrize("p", MODULI)
def test_oracle_u64_against_python_integers(p):
    rng = np.random.default_rng(p % 9973)
    A = rng.integers(0, p, (7, 19), dtype=np.uint64)
    B = rng.integers(0, p, (19, 5), dtype=np.uint64)
    C = rng.integers(0, p, (7, 5), dtype=np.uint64)
    for op in (0, 1, 2):
        assert np.array_equal(O.gemm_u64(p, A, B, C, op), _exact(p, A, B, C, op))
    full = np.full((4, 33), p - 1, np.uint64)  # the largest products
    assert np.array_equal(O.gemm_u64(p, full, full.T.copy()), _exact(p, full, full.T.copy(), np.zeros((4, 4)), 0))


@pytest.mark.skipif(not O.ref_available(), reason="reference CPU engine not built here")
@pytest.mark.parametrize("p", MODULI)
def test_oracle_u64_matches_reference(p):
    rng = np.random.default_rng(p % 7919)
    A = rng.integers(0, p, (31, 70), dtype=np.uint64)
    B = rng.integers(0, p, (70, 23), dtype=np.uint64)
    C = rng.integers(0, p, (31, 23), dtype=np.uint64)
    for op in (0, 1, 2):
        assert np.array_equal(O.gemm_u64(p, A, B, C, op), O.ref_gemm_u64(p, A, B, C, op))


def test_oracle_u64_reproduces_golden():
    for g in GOLD["gemm_u64"]:
        m, n, k, p = g["m"], g["n"], g["k"], g["p"]
        rng = np.random.default_rng(g["seed"])
        A = rng.integers(0, p, (m, k), dtype=np.uint64)
        B = rng.integers(0, p, (k, n), dtype=np.uint64)
        C = rng.integers(0, p, (m, n), dtype=np.uint64)
        R = O.gemm_u64(p, A, B, C, g["op"])
        assert "0x%016x" % O.fnv_matrix(R.view(np.uint32).reshape(m, 2 * n)) == g["fnv"]
