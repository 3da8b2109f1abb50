"""Parity of the device elimination over F_p (through the C ABI) with the oracle.

RREF, pivots, rank, determinant, kernel basis, inverse and solve are unique
functions of the input, so every comparison is exact (tolerance zero).  The
small cases compare against oracle/oracle.c; the full-size configuration
(4096 x 4096, rank 3900, p = 2^31 - 19) compares checksums with the golden
fixture produced by the reference's own engine (tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle as O
from hacs_b200 import HmeError, gen

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
PRIMES = [2, 3, 13, 251, 65521, 16777213, 2147483629, 4294967291]


def _rand(rng, shape, p):
    return rng.integers(0, p, shape, dtype=np.uint64).astype(np.uint32)


def _ranked(rng, m, n, r, p):
    return O.gemm(p, _rand(rng, (m, r), p), _rand(rng, (r, n), p))


@pytest.mark.parametrize("p", PRIMES)
def test_rref_random_shapes(engine, p):
    rng = np.random.default_rng(p % 1009)
    cases = [(1, 1, 1), (5, 9, 3), (40, 30, 30), (64, 64, 64), (130, 200, 70), (257, 100, 100), (100, 257, 60)]
    for (m, n, r) in cases:
        A = _ranked(rng, m, n, r, p)
        R1, p1 = engine.rref(p, A)
        R2, p2 = O.rref(p, A)
        assert np.array_equal(p1, p2), (p, m, n)
        assert np.array_equal(R1, R2), (p, m, n)


def test_rref_edge_cases(engine):
    p = 65521
    rng = np.random.default_rng(4)
    Z = np.zeros((33, 47), np.uint32)
    R, piv = engine.rref(p, Z)
    assert len(piv) == 0 and not R.any()
    I = np.eye(70, dtype=np.uint32)
    R, piv = engine.rref(p, I)
    assert np.array_equal(R, I) and list(piv) == list(range(70))
    A = _rand(rng, (90, 120), p)
    A[:, ::3] = 0           # zero columns are never pivots
    A[10] = A[3]            # a repeated row
    R1, p1 = engine.rref(p, A)
    R2, p2 = O.rref(p, A)
    assert np.array_equal(R1, R2) and np.array_equal(p1, p2)
    one = np.array([[0, 0, 5, 7]], np.uint32)
    R, piv = engine.rref(p, one)
    assert list(piv) == [2] and R[0, 2] == 1


@pytest.mark.parametrize("case", GOLD["rref"], ids=lambda c: f"rref{c['m']}x{c['n']}r{c['rank_target']}")
def test_rref_golden(engine, case):
    L, R = gen.ranked_factors(case["m"], case["n"], case["rank_target"], case["p"])
    A = engine.gemm(case["p"], L, R)
    assert gen.fnv_matrix(A) == int(case["input_fnv"], 16)
    Rr, piv = engine.rref(case["p"], A)
    assert list(piv) == case["pivots"]
    assert gen.fnv_matrix(Rr) == int(case["rref_fnv"], 16)


def test_rref_invariant_under_tuning(engine):
    p = 2147483629
    rng = np.random.default_rng(8)
    A = _ranked(rng, 300, 280, 250, p)
    want, wp = O.rref(p, A)
    try:
        for (panel, rpc, ctas) in [(8, 4, 0), (32, 16, 3), (128, 256, 0), (64, 1, 7), (1, 32, 0)]:
            engine.set_elim_options(panel, rpc, ctas, 16 if panel < 64 else 128)
            R, piv = engine.rref(p, A)
            assert np.array_equal(R, want) and np.array_equal(piv, wp), (panel, rpc, ctas)
    finally:
        engine.set_elim_options()


@pytest.mark.parametrize("p", [13, 65521, 2147483629])
def test_rank_profile_and_det(engine, p):
    rng = np.random.default_rng(p % 101)
    for n in (1, 2, 7, 33, 128, 200):
        A = _rand(rng, (n, n), p)
        assert engine.det(p, A) == O.det(p, A)
        _, piv = O.rref(p, A)
        assert np.array_equal(engine.column_rank_profile(p, A), piv)
    S = _ranked(rng, 150, 150, 120, p)
    assert engine.det(p, S) == 0
    R, piv, d = engine.rref_det(p, S)
    R2, p2 = O.rref(p, S)
    assert d == 0 and np.array_equal(R, R2) and np.array_equal(piv, p2)
    A, B = _rand(rng, (90, 90), p), _rand(rng, (90, 90), p)
    assert engine.det(p, engine.gemm(p, A, B)) == engine.det(p, A) * engine.det(p, B) % p


def test_kernel_inverse_solve(engine):
    p = 2147483629
    rng = np.random.default_rng(12)
    A = _ranked(rng, 60, 90, 45, p)
    K = engine.kernel_basis(p, A)
    R, piv = O.rref(p, A)
    assert np.array_equal(K, O.kernel_basis(p, R, piv))
    assert not engine.gemm(p, A, K.T.copy()).any()
    M = _rand(rng, (77, 77), p)
    X = engine.inverse(p, M)
    assert np.array_equal(X, O.inverse(p, M))
    assert engine.inverse(p, _ranked(rng, 40, 40, 39, p)) is None
    B = _rand(rng, (120, 50), p)
    Xs = _rand(rng, (50, 7), p)
    Y = engine.gemm(p, B, Xs)
    assert np.array_equal(engine.solve_multi_rhs(p, B, Y), Xs)
    Y[3, 2] = (Y[3, 2] + 1) % p
    assert engine.solve_multi_rhs(p, B, Y) is None


def test_composite_modulus_refused(engine):
    with pytest.raises(HmeError) as e:
        engine.rref(65536, np.ones((4, 4), np.uint32))
    assert "not prime" in str(e.value)


def test_rref_device_pointer(engine):
    import torch

    p = 65521
    rng = np.random.default_rng(21)
    A = _ranked(rng, 200, 180, 150, p)
    dA = torch.from_numpy(A.view(np.int32)).cuda()
    engine.use_own_stream()
    piv = engine.rref_dev(p, dA)
    R2, p2 = O.rref(p, A)
    assert np.array_equal(piv, p2)
    assert np.array_equal(dA.cpu().numpy().view(np.uint32), R2)


def test_rref_config2_full_size_golden(engine):
    """Config 2: RankedMatrix(4096, 4096, 3900, 2^31 - 19); RREF, pivots and det
    bit-exact against the reference engine's (checksums from the golden file)."""
    c = GOLD.get("config2")
    if c is None:
        pytest.skip("golden file built without the full-size cases")
    p = c["p"]
    L, R = gen.ranked_factors(c["m"], c["n"], c["rank_target"], p)
    A = engine.gemm(p, L, R)
    assert gen.fnv_matrix(A) == int(c["input_fnv"], 16)
    Rr, piv, d = engine.rref_det(p, A)
    assert len(piv) == c["rank"] == 3900
    assert gen.fnv_matrix(piv.reshape(1, -1)) == int(c["pivots_fnv"], 16)
    assert gen.fnv_matrix(Rr) == int(c["rref_fnv"], 16)
    assert d == c["det"] == 0


@pytest.mark.parametrize("p", [3, 65521, 2147483629, 4294967291])
def test_panel_kernels_agree(engine, p):
    """The thread-block-cluster panel kernel (DSMEM exchange, one cluster) and
    the cooperative grid kernel give the oracle's RREF and pivots, on shapes
    that take 1, 2, 4, 8 and 16 CTAs per cluster and on one whose panel does
    not fit a cluster (the automatic choice falls back to the grid kernel)."""
    rng = np.random.default_rng(p % 977)
    cases = [(100, 80, 50), (400, 100, 90), (600, 300, 200), (1500, 700, 690), (3000, 200, 150), (5000, 130, 128)]
    try:
        for (m, n, r) in cases:
            A = _ranked(rng, m, n, r, p)
            R2, p2 = O.rref(p, A)
            for mode in (2, 1, 0):
                engine.set_panel_kernel(mode)
                R1, p1 = engine.rref(p, A)
                assert np.array_equal(p1, p2), (p, m, n, mode)
                assert np.array_equal(R1, R2), (p, m, n, mode)
        # 20000 active rows x 64 columns: more than one cluster's shared memory
        A = _ranked(rng, 20000, 64, 40, p)
        engine.set_panel_kernel(2)
        with pytest.raises(HmeError):
            engine.rref(p, A)
        engine.set_panel_kernel(0)
        R1, p1 = engine.rref(p, A)
        R2, p2 = O.rref(p, A)
        assert np.array_equal(p1, p2) and np.array_equal(R1, R2)
    finally:
        engine.set_panel_kernel(0)


@pytest.mark.parametrize("ell,k", [(2, 16), (3, 10), (2, 31), (5, 3)])
def test_panel_kernels_agree_ring(engine, ell, k):
    """Both panel kernels and the automatic mode (top-block path first) in the
    ring mode (minimal-valuation pivots) give the reference's Howell form and
    Smith valuations."""
    rng = np.random.default_rng(ell * 100 + k)
    q = ell ** k
    A = rng.integers(0, q, (300, 260), dtype=np.uint64).astype(np.uint32)
    A[:, 5] = ((A[:, 5].astype(np.uint64) * ell) % q).astype(np.uint32)
    want_h = O.howell(ell, k, A)
    want_s = O.smith(ell, k, A)
    try:
        for mode in (2, 1, 0):
            engine.set_panel_kernel(mode)
            H, piv, pv = engine.howell(ell, k, A)
            assert np.array_equal(H, want_h[0]) and np.array_equal(piv, want_h[1]), (ell, k, mode)
            assert np.array_equal(engine.smith(ell, k, A), want_s), (ell, k, mode)
    finally:
        engine.set_panel_kernel(0)


@pytest.mark.parametrize("p", [2, 3, 65521, 2147483629, 4294967291])
def test_top_block_path(engine, p):
    """Over a field, a panel whose top rows factor with non-zero diagonal
    entries is settled without a search (its pivots are those rows in order,
    the rows below take x U^-1); a zero on that diagonal sends the panel to the
    searching kernel.  Both kinds of panel, at several panel widths, give the
    oracle's RREF and pivots, and the context's counters see both paths."""
    rng = np.random.default_rng(p % 1013)
    b0, s0 = engine.elim_panel_stats()
    cases = []
    cases.append(_rand(rng, (300, 300), p))                 # generic: every panel settled by its top block
    cases.append(_ranked(rng, 260, 300, 200, p))            # rank-deficient: the last panels search
    A = _rand(rng, (200, 190), p)
    A[4, :] = A[2, :]                                       # step 4 of panel 0 meets a zero: search
    A[0, 0] = 0                                             # and the very first entry is zero
    cases.append(A)
    A = _rand(rng, (150, 400), p)
    A[70:90, 64:128] = 0                                    # a zero block inside panel 1's top rows
    cases.append(A)
    cases.append(_rand(rng, (40, 300), p))                  # fewer active rows than the panel width
    try:
        for panel in (0, 8, 33, 100, 128):
            engine.set_elim_options(panel, 0, 0, 0)
            for A in cases:
                R1, p1 = engine.rref(p, A)
                R2, p2 = O.rref(p, A)
                assert np.array_equal(p1, p2), (p, A.shape, panel)
                assert np.array_equal(R1, R2), (p, A.shape, panel)
            n = 97
            M = _rand(rng, (n, n), p)
            assert engine.det(p, M) == O.det(p, M), (p, panel)
    finally:
        engine.set_elim_options()
    b1, s1 = engine.elim_panel_stats()
    assert s1 > s0, (s0, s1)
    if p >= 256:
        assert b1 > b0, (b0, b1)
    else:  # small fields go straight to the search
        assert b1 == b0, (b0, b1)


def test_top_block_path_ring_and_forced_modes(engine):
    """The ring forms (minimal-valuation pivots over Z/ell^k) and the forced kernel
    modes never take the top-block path; the ring forms stay equal to the
    oracle's, also on inputs whose leading minors are all units."""
    rng = np.random.default_rng(5)
    b0, _ = engine.elim_panel_stats()
    for ell, k in ((2, 16), (3, 10)):
        q = ell ** k
        Lw = np.tril(rng.integers(0, q, (200, 180), dtype=np.uint64), -1)
        Up = np.triu(rng.integers(0, q, (180, 180), dtype=np.uint64), 1)
        units = rng.integers(1, q, 180, dtype=np.uint64)
        units = np.where(units % ell == 0, units + 1, units) % q
        Lw[np.arange(180), np.arange(180)] = 1
        Up[np.arange(180), np.arange(180)] = units
        A = O.gemm(q, Lw.astype(np.uint32), Up.astype(np.uint32))
        R = rng.integers(0, q, (150, 170), dtype=np.uint64).astype(np.uint32)
        for M in (A, R):
            H, piv, pv = engine.howell(ell, k, M)
            want = O.howell(ell, k, M)
            assert np.array_equal(H, want[0]) and np.array_equal(piv, want[1]), (ell, k)
    b1, _ = engine.elim_panel_stats()
    assert b1 == b0
    b0, _ = engine.elim_panel_stats()
    try:
        for mode in (1, 2, 3):
            engine.set_panel_kernel(mode)
            B = _rand(rng, (150, 150), 65521)
            R1, p1 = engine.rref(65521, B)
            R2, p2 = O.rref(65521, B)
            assert np.array_equal(R1, R2) and np.array_equal(p1, p2)
    finally:
        engine.set_panel_kernel(0)
    b1, _ = engine.elim_panel_stats()
    assert b1 == b0
