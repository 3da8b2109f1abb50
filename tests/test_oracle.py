"""CPU tests: the oracle restatement pinned to the reference's golden fixtures
(tests/golden/golden.json, generated from the reference's own engine by
tests/golden/make_golden.py), the reference's known answers, and -- where the
reference library was built here -- direct cross-checks on fresh inputs."""
import json
import os

import numpy as np
import pytest

import oracle as O
from hacs_b200 import gen

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def fnv(M):
    return "0x%016x" % O.fnv_matrix(np.ascontiguousarray(M, dtype=np.uint32))


def test_generator_matches_oracle_generator():
    for (r, c, p, salt) in [(7, 9, 65521, 1), (64, 33, 2147483629, 2), (1, 1000, 13, 0x21)]:
        assert np.array_equal(gen.engine_matrix(r, c, p, salt), O.engine_matrix(r, c, p, salt))


@pytest.mark.parametrize("case", GOLD["gemm"], ids=lambda c: f"gemm{c['n']}x{c['k']}p{c['p']}")
def test_oracle_gemm_golden(case):
    if case["n"] * case["n"] * case["k"] > 3e8:
        pytest.skip("large golden case covered on the GPU")
    A = gen.engine_matrix(case["n"], case["k"], case["p"], 1)
    B = gen.engine_matrix(case["k"], case["n"], case["p"], 2)
    assert fnv(O.gemm(case["p"], A, B)) == case["fnv"]


@pytest.mark.parametrize("case", GOLD["rref"], ids=lambda c: f"rref{c['m']}x{c['n']}r{c['rank_target']}")
def test_oracle_rref_golden(case):
    L, R = gen.ranked_factors(case["m"], case["n"], case["rank_target"], case["p"])
    A = O.gemm(case["p"], L, R)
    assert fnv(A) == case["input_fnv"]
    Rr, piv = O.rref(case["p"], A)
    assert len(piv) == case["rank"] and list(piv) == case["pivots"]
    assert fnv(Rr) == case["rref_fnv"]


@pytest.mark.parametrize("case", GOLD["ring"], ids=lambda c: f"ring{c['ell']}^{c['k']}n{c['n']}")
def test_oracle_howell_smith_golden(case):
    M, e = gen.planted_udv(case["n"], case["ell"], case["k"], case["salt"])
    assert fnv(M) == case["input_fnv"] and list(e) == case["planted_e"]
    H, piv, pv = O.howell(case["ell"], case["k"], M)
    assert len(piv) == case["h"] and list(piv) == case["pivots"] and list(pv) == case["pivot_v"]
    assert fnv(H) == case["howell_fnv"]
    sig = O.smith(case["ell"], case["k"], M)
    assert list(sig) == case["sigma"]
    assert list(sig) == sorted(x for x in case["planted_e"] if x < case["k"])  # planted known answer


def test_oracle_known_answers_z4():
    k = GOLD["known"]
    H, piv, pv = O.howell(2, 2, np.array([[2, 1]], np.uint32))
    assert H.tolist() == k["howell_z4_row_2_1"]["H"] == [[2, 1], [0, 2]]
    assert pv.tolist() == [1, 1]
    H, piv, pv = O.howell(2, 2, np.array([[2], [1]], np.uint32))
    assert H.tolist() == k["howell_z4_col_2_1"]["H"] and pv.tolist() == [0]
    assert O.smith(2, 2, np.array([[2], [1]], np.uint32)).tolist() == k["smith_z4_col_2_1"] == [0]


def test_oracle_howell_at_k1_is_rref_without_zero_rows():
    rng = np.random.default_rng(5)
    p = 13
    A = rng.integers(0, p, (9, 12)).astype(np.uint32)
    A[3] = (2 * A[1] + A[2]) % p
    H, piv, pv = O.howell(p, 1, A)
    R, rp = O.rref(p, A)
    assert np.array_equal(H, R[: len(rp)]) and np.array_equal(piv, rp) and not pv.any()


def test_oracle_det_product_rule_and_rank():
    rng = np.random.default_rng(11)
    p = 2147483629
    for n in (1, 2, 5, 17, 40):
        A = rng.integers(0, p, (n, n), dtype=np.uint64).astype(np.uint32)
        B = rng.integers(0, p, (n, n), dtype=np.uint64).astype(np.uint32)
        AB = O.gemm(p, A, B)
        assert O.det(p, AB) == O.det(p, A) * O.det(p, B) % p
    L, R = gen.ranked_factors(30, 30, 20, p)
    assert O.det(p, O.gemm(p, L, R)) == 0


def test_oracle_inverse_and_solve():
    rng = np.random.default_rng(2)
    p = 65521
    A = rng.integers(0, p, (20, 20)).astype(np.uint32)
    X = O.inverse(p, A)
    assert X is not None
    assert np.array_equal(O.gemm(p, A, X), np.eye(20, dtype=np.uint32))
    B = rng.integers(0, p, (30, 12)).astype(np.uint32)
    Xs = rng.integers(0, p, (12, 5)).astype(np.uint32)
    Y = O.gemm(p, B, Xs)
    assert np.array_equal(O.solve(p, B, Y), Xs)
    Y[0, 0] = (Y[0, 0] + 1) % p  # a right-hand side outside the span (B has full column rank 12 < 30)
    assert O.solve(p, B, Y) is None


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_oracle_matches_reference_on_fresh_inputs():
    rng = np.random.default_rng(99)
    for p in (2, 3, 65521, 2147483629, 4294967291):
        A = rng.integers(0, p, (37, 53), dtype=np.uint64).astype(np.uint32)
        B = rng.integers(0, p, (53, 29), dtype=np.uint64).astype(np.uint32)
        Cm = rng.integers(0, p, (37, 29), dtype=np.uint64).astype(np.uint32)
        for op in range(3):
            assert np.array_equal(O.gemm(p, A, B, Cm, op), O.ref_gemm(p, A, B, Cm, op))
    for (ell, k) in [(2, 16), (3, 10), (5, 3)]:
        q = ell ** k
        A = (rng.integers(0, q, (25, 31)) * rng.choice([1, ell, ell * ell], (25, 31))) % q
        A = A.astype(np.uint32)
        for x, y in zip(O.howell(ell, k, A), O.ref_elim_howell(ell, k, A)):
            assert np.array_equal(x, y)


def test_oracle_planted_mistake_is_caught():
    """Negative control: a one-entry perturbation of the input changes the checksum."""
    case = GOLD["rref"][0]
    L, R = gen.ranked_factors(case["m"], case["n"], case["rank_target"], case["p"])
    A = O.gemm(case["p"], L, R)
    A[5, 7] = (A[5, 7] + 1) % case["p"]
    Rr, piv = O.rref(case["p"], A)
    assert fnv(Rr) != case["rref_fnv"]


def test_job_stream_golden_pins_restatement():
    """The config-4 golden file (the reference engine's rank and C checksum of
    every job) agrees with the oracle's C restatement on a strided sample of
    the stream's smaller jobs."""
    import json

    from hacs_b200 import gen

    path = os.path.join(os.path.dirname(__file__), "golden", "jobs10000.json")
    d = json.load(open(path))
    assert d["n_jobs"] == len(d["rank"]) == len(d["c_fnv"]) == 10000
    s, fam, p, sa, sb = gen.job_stream(10000)
    checked = 0
    for j in range(0, 10000, 97):
        n = int(s[j])
        if n > 160:
            continue
        A = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sa[j]))
        B = gen.job_matrix(n, n, int(p[j]), int(fam[j]), int(sb[j]))
        Cm = O.gemm(int(p[j]), A, B)
        assert O.fnv_matrix(Cm) == int(d["c_fnv"][j], 16), j
        assert len(O.rref(int(p[j]), Cm)[1]) == d["rank"][j], j
        checked += 1
    assert checked >= 40
