"""Parity of the device Howell and Smith forms over Z/ell^k (through the C ABI)
with the oracle and with the reference's golden fixtures.  Both forms are
unique functions of the input: comparisons are exact."""
import json
import os

import numpy as np
import pytest

import oracle as O
from hacs_b200 import HmeError, gen

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
RINGS = [(2, 1), (2, 2), (2, 16), (3, 1), (3, 10), (5, 3), (2, 31), (3, 19), (65521, 2)]


def _structured(rng, m, n, ell, k):
    q = ell ** k
    A = rng.integers(0, q, (m, n), dtype=np.uint64)
    scale = rng.choice([1, ell, ell * ell % q, ell ** min(k, 3) % q], (m, n)).astype(np.uint64)
    A = (A * scale) % q
    A[rng.random((m, n)) < 0.2] = 0
    return A.astype(np.uint32)


@pytest.mark.parametrize("ell,k", RINGS)
def test_howell_matches_oracle(engine, ell, k):
    rng = np.random.default_rng(ell * 31 + k)
    for (m, n) in [(1, 2), (3, 3), (6, 6), (12, 9), (9, 14), (40, 33), (70, 90)]:
        A = _structured(rng, m, n, ell, k)
        H1, p1, v1 = engine.howell(ell, k, A)
        H2, p2, v2 = O.howell(ell, k, A)
        assert np.array_equal(p1, p2) and np.array_equal(v1, v2), (ell, k, m, n)
        assert np.array_equal(H1, H2), (ell, k, m, n)


@pytest.mark.parametrize("ell,k", RINGS)
def test_smith_matches_oracle(engine, ell, k):
    rng = np.random.default_rng(ell * 17 + k)
    for (m, n) in [(1, 1), (4, 7), (20, 20), (33, 25), (64, 64), (100, 80)]:
        A = _structured(rng, m, n, ell, k)
        assert np.array_equal(engine.smith(ell, k, A), O.smith(ell, k, A)), (ell, k, m, n)


def test_known_answers_z4(engine):
    H, piv, pv = engine.howell(2, 2, np.array([[2, 1]], np.uint32))
    assert H.tolist() == [[2, 1], [0, 2]] and piv.tolist() == [0, 1] and pv.tolist() == [1, 1]
    H, piv, pv = engine.howell(2, 2, np.array([[2], [1]], np.uint32))
    assert H.tolist() == [[1]] and pv.tolist() == [0]
    assert engine.smith(2, 2, np.array([[2], [1]], np.uint32)).tolist() == [0]
    assert engine.invariant_factors(2, 2, np.array([[2], [1]], np.uint32)).tolist() == [2]


def test_howell_edge_cases(engine):
    z = np.zeros((5, 7), np.uint32)
    H, piv, pv = engine.howell(3, 4, z)
    assert H.shape[0] == 0
    I = np.eye(9, dtype=np.uint32)
    H, piv, pv = engine.howell(2, 16, I)
    assert np.array_equal(H, I) and not pv.any()
    assert len(engine.smith(2, 16, z)) == 0
    with pytest.raises(HmeError):
        engine.howell(2, 4, np.array([[16]], np.uint32))  # not canonical mod 2^4
    with pytest.raises(HmeError):
        engine.smith(4, 2, np.array([[1]], np.uint32))    # ell not prime


def test_howell_uniqueness_under_row_operations(engine):
    """The Howell form is a function of the row span: unchanged under row
    permutation, unimodular left multiplication and appended span rows."""
    rng = np.random.default_rng(9)
    ell, k = 3, 10
    q = ell ** k
    A = _structured(rng, 30, 40, ell, k)
    base = engine.howell(ell, k, A)
    perm = A[rng.permutation(30)]
    U = np.eye(30, dtype=np.uint64)
    for _ in range(50):
        i, j = rng.choice(30, 2, replace=False)
        U[i] = (U[i] + int(rng.integers(-5, 6)) % q * U[j]) % q
    UA = engine.gemm(q, U.astype(np.uint32), A)
    extra = np.vstack([A, engine.gemm(q, rng.integers(0, q, (5, 30), dtype=np.uint64).astype(np.uint32), A)])
    for B in (perm, UA, extra):
        got = engine.howell(ell, k, B)
        for x, y in zip(got, base):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("case", GOLD["ring"], ids=lambda c: f"ring{c['ell']}^{c['k']}n{c['n']}")
def test_ring_golden(engine, case):
    M, e = gen.planted_udv(case["n"], case["ell"], case["k"], case["salt"])
    H, piv, pv = engine.howell(case["ell"], case["k"], M)
    assert list(piv) == case["pivots"] and list(pv) == case["pivot_v"]
    assert gen.fnv_matrix(H) == int(case["howell_fnv"], 16)
    assert list(engine.smith(case["ell"], case["k"], M)) == case["sigma"]


@pytest.mark.parametrize("key", ["2^16", "3^10"])
def test_config3_full_size_golden(engine, key):
    """Config 3: planted U*D*V, 2048 x 2048: Howell over Z/2^16 and Smith over
    Z/3^10 (and the other form of each ring) bit-exact against the reference
    engine's, and sigma equal to the planted valuations."""
    c = GOLD.get("config3", {}).get(key)
    if c is None:
        pytest.skip("golden file built without the full-size cases")
    M, e = gen.planted_udv(c["n"], c["ell"], c["k"], c["salt"])
    assert gen.fnv_matrix(M) == int(c["input_fnv"], 16)
    sig = engine.smith(c["ell"], c["k"], M)
    assert list(sig) == c["sigma"] == sorted(int(x) for x in e if x < c["k"])
    H, piv, pv = engine.howell(c["ell"], c["k"], M)
    assert len(piv) == c["h"]
    assert gen.fnv_matrix(piv.reshape(1, -1)) == int(c["pivots_fnv"], 16)
    assert gen.fnv_matrix(pv.reshape(1, -1)) == int(c["pivot_v_fnv"], 16)
    assert gen.fnv_matrix(H) == int(c["howell_fnv"], 16)
