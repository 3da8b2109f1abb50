"""The u64-residue GEMM (hme_gemm_u64 / hme_gemm_u64_dev, through the C ABI)
bit-exact against the oracle and the reference's golden checksums: moduli
from 2 to 2^64 - 59 (the narrow u32 route below 2^32, Montgomery for odd
p < 2^63, the wide reduction for even p and p >= 2^63), Set / Add / Sub,
ragged shapes, k = 0, inner dimensions across the limb GEMM's chunk sizes,
operands of all p - 1."""
import json
import os

import numpy as np
import pytest

import hacs_b200
import oracle as O

pytestmark = pytest.mark.gpu

MODULI = [2, 251, 134217757, 4294967291, 4294967311, 1099511627776, 10**12, 2305843009213693951,
          9223372036854775783, 9223372036854775837, 18446744073709551557]


def _rand(rng, p, shape):
    return rng.integers(0, p, shape, dtype=np.uint64)


@pytest.mark.parametrize("p", MODULI)
def test_gemm_u64_host_matches_oracle(engine, p):
    rng = np.random.default_rng(p % 10007)
    for m, n, k in [(1, 1, 1), (37, 53, 20), (128, 128, 128), (200, 70, 513), (65, 300, 1)]:
        A, B, C = _rand(rng, p, (m, k)), _rand(rng, p, (k, n)), _rand(rng, p, (m, n))
        for op in (hacs_b200.SET, hacs_b200.ADD, hacs_b200.SUB):
            got = engine.gemm_u64(p, A, B, C, op)
            assert np.array_equal(got, O.gemm_u64(p, A, B, C, op)), (p, m, n, k, op)


@pytest.mark.parametrize("p", [4294967311, 2305843009213693951, 18446744073709551557, 9223372036854775837])
def test_gemm_u64_extremes(engine, p):
    """All-(p-1) operands (the largest sum the residue system must hold), a long
    inner dimension, and k = 0."""
    full_a = np.full((40, 3000), p - 1, np.uint64)
    full_b = np.full((3000, 24), p - 1, np.uint64)
    assert np.array_equal(engine.gemm_u64(p, full_a, full_b), O.gemm_u64(p, full_a, full_b))
    C = np.full((5, 6), 7, np.uint64)
    empty_a, empty_b = np.zeros((5, 0), np.uint64), np.zeros((0, 6), np.uint64)
    assert (engine.gemm_u64(p, empty_a, empty_b, C, hacs_b200.SET) == 0).all()
    assert (engine.gemm_u64(p, empty_a, empty_b, C, hacs_b200.ADD) == 7).all()


@pytest.mark.parametrize("p", [134217757, 2305843009213693951, 18446744073709551557])
def test_gemm_u64_dev_padded_views(engine, p):
    import torch

    rng = np.random.default_rng(5)
    A, B, C = _rand(rng, p, (90, 77)), _rand(rng, p, (77, 45)), _rand(rng, p, (90, 45))
    Ab = torch.zeros((90, 80), dtype=torch.int64, device="cuda")
    Bb = torch.zeros((77, 50), dtype=torch.int64, device="cuda")
    Cb = torch.zeros((90, 49), dtype=torch.int64, device="cuda")
    Ab[:, :77] = torch.from_numpy(A.view(np.int64))
    Bb[:, :45] = torch.from_numpy(B.view(np.int64))
    Cb[:, :45] = torch.from_numpy(C.view(np.int64))
    engine.gemm_u64_dev(p, Ab[:, :77], Bb[:, :45], Cb[:, :45], hacs_b200.SUB)
    engine.sync()
    got = Cb.cpu().numpy().view(np.uint64)
    assert np.array_equal(got[:, :45], O.gemm_u64(p, A, B, C, hacs_b200.SUB))
    assert (got[:, 45:] == 0).all()


def test_gemm_u64_reproduces_reference_golden(engine):
    G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "level12.json")))
    for g in G["gemm_u64"]:
        m, n, k, p = g["m"], g["n"], g["k"], g["p"]
        rng = np.random.default_rng(g["seed"])
        A, B, C = _rand(rng, p, (m, k)), _rand(rng, p, (k, n)), _rand(rng, p, (m, n))
        R = engine.gemm_u64(p, A, B, C, g["op"])
        assert "0x%016x" % O.fnv_matrix(R.view(np.uint32).reshape(m, 2 * n)) == g["fnv"], g
