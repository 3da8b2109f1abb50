"""The scheduler on the GPU: every GEMM variant bit-exact, the MLP's GPU
gradients against the CPU reference, BF16 inference against the reference's
bf16 emulation, training, the learned plan routing GEMMs without changing a
value, and the trained network's gain over the method without it."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
from hacs_b200 import ADD, SET, SUB, _lib, sched
from oracle import mlp_ref as R

pytestmark = pytest.mark.gpu


def _dev(M):
    import torch

    return torch.from_numpy(np.ascontiguousarray(M).view(np.int32)).cuda()


@pytest.mark.parametrize("p", [13, 65521, 16777213, 2147483629, 4294967291])
def test_every_variant_bit_exact(engine, p):
    rng = np.random.default_rng(p % 1000)
    L = _lib.lib()
    for (m, k, n) in [(1, 1, 1), (16, 16, 16), (33, 17, 65), (128, 128, 128), (300, 257, 200)]:
        A = rng.integers(0, p, (m, k), dtype=np.uint64).astype(np.uint32)
        B = rng.integers(0, p, (k, n), dtype=np.uint64).astype(np.uint32)
        C0 = rng.integers(0, p, (m, n), dtype=np.uint64).astype(np.uint32)
        for op in (SET, ADD, SUB):
            want = O.gemm(p, A, B, C0, op)
            for v in range(L.hme_gemm_variant_count()):
                dA, dB, dC = _dev(A), _dev(B), _dev(C0)
                _lib.check(L.hme_gemm_u32_dev_variant(engine._h, v, p, m, n, k, dA.data_ptr(), k, dB.data_ptr(), n,
                                                      dC.data_ptr(), n, op))
                engine.sync()
                assert np.array_equal(dC.cpu().numpy().view(np.uint32), want), (p, m, k, n, op, v)


def test_mlp_gradient_matches_cpu_reference(engine):
    rng = np.random.default_rng(1)
    mlp = sched.MLP(engine, seed=3)
    w = rng.normal(0, 0.2, mlp.n_params).astype(np.float32)
    mlp.set_params(w)
    X = rng.normal(0, 1, (300, 5)).astype(np.float32)
    Y = rng.normal(0, 1, (300, 4)).astype(np.float32)
    loss, g = mlp.loss_grad(X, Y)
    ref_loss, ref_g = R.loss_grad(w.astype(np.float64), X, Y)
    assert abs(loss - ref_loss) <= 1e-5 * max(1.0, abs(ref_loss))  # fp32 tolerance
    assert np.max(np.abs(g - ref_g)) <= 1e-4 * np.max(np.abs(ref_g)) + 1e-7


def test_mlp_bf16_inference_matches_reference_emulation(engine):
    rng = np.random.default_rng(2)
    mlp = sched.MLP(engine, seed=4)
    w = mlp.get_params()
    X = rng.normal(0, 1, (500, 5)).astype(np.float32)
    got = mlp.predict_normalised(X)
    want = R.forward_bf16(w, X)
    scale = np.max(np.abs(want)) + 1e-6
    assert np.max(np.abs(got - want)) <= 1e-2 * scale  # bf16 tolerance (8-bit mantissa, fp32 accumulation)
    full, _ = R.forward(w, X)
    assert np.max(np.abs(got - full)) <= 5e-2 * scale


def test_mlp_training_reduces_loss(engine):
    rng = np.random.default_rng(3)
    X = rng.normal(0, 1, (4000, 5)).astype(np.float32)
    Y = np.stack([X.sum(1), X[:, 0] * X[:, 1], np.maximum(X[:, 2], 0), -X[:, 3] + 0.5 * X[:, 4]], 1)
    Y = ((Y - Y.mean(0)) / Y.std(0)).astype(np.float32)
    mlp = sched.MLP(engine, seed=9)
    before, _ = mlp.loss_grad(X, Y)
    after = mlp.train_normalised(X, Y, epochs=60, batch=256, lr=3e-3)
    assert after < 0.1 * before


def test_learned_plan_routes_gemms_without_changing_values(engine):
    """A network whose outputs prefer the 32 x 32 CUDA-core variant: after
    hme_sched_plan, policy 1 sends the planned shapes there; results unchanged."""
    mlp = sched.MLP(engine, seed=1)
    w = np.zeros(mlp.n_params, np.float32)
    w[-4:] = [1.0, 1.0, 0.0, 1.0]  # output biases: variant 2 has the smallest predicted time
    mlp.set_params(w)
    p = 2147483629
    shapes = np.array([[p, 48, 40, 56]], np.uint32)
    assert list(mlp.plan(shapes)) == [2]
    L = _lib.lib()
    rng = np.random.default_rng(5)
    A = rng.integers(0, p, (48, 56), dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, p, (56, 40), dtype=np.uint64).astype(np.uint32)
    try:
        _lib.check(L.hme_ctx_set_sched_policy(engine._h, 1))
        engine.set_timing(True)
        engine.timing_reset()
        got = engine.gemm(p, A, B)
        _, simt_launches = engine.kernel_time("simt_gemm")
        _, tensor_launches = engine.kernel_time("limb_gemm")
    finally:
        engine.set_timing(False)
        _lib.check(L.hme_ctx_set_sched_policy(engine._h, 0))
    assert simt_launches == 1 and tensor_launches == 0
    assert np.array_equal(got, O.gemm(p, A, B))


def test_learned_rank_plan_routes_rank_rounds_without_changing_ranks(engine):
    """A rank-planner network whose outputs prefer schedule 2 (the CUDA-core
    trailing update, last panel up to 128 columns): after hme_sched_plan_rank, policy 1 runs
    the planned jobs' trailing updates on CUDA cores and no grouped limb GEMM
    in their rank rounds; the rank is unchanged."""
    import torch

    mlp = sched.MLP(engine, seed=1)
    w = np.zeros(mlp.n_params, np.float32)
    w[-4:] = [1.0, 1.0, 0.0, 1.0]
    mlp.set_params(w)
    p, m, n, r = 2147483629, 200, 300, 120
    assert list(mlp.plan_rank(np.array([[p, m, n, r]], np.uint32))) == [2]
    rng = np.random.default_rng(8)
    A = rng.integers(0, p, (m, r), dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, p, (r, n), dtype=np.uint64).astype(np.uint32)
    jobs = [{"p": p, "A": _dev(A), "B": _dev(B), "C": torch.zeros((m, n), dtype=torch.int32, device="cuda")}]
    L = _lib.lib()
    try:
        _lib.check(L.hme_ctx_set_sched_policy(engine._h, 1))
        engine.set_timing(True)
        engine.timing_reset()
        ranks = engine.batch_gemm_rank_dev(jobs)
        _, simt_launches = engine.kernel_time("batch_simt_update")
    finally:
        engine.set_timing(False)
        _lib.check(L.hme_ctx_set_sched_policy(engine._h, 0))
    assert simt_launches > 0
    assert list(ranks) == [len(O.rref(p, O.gemm(p, A, B))[1])] == [r]


@pytest.mark.skipif(not os.path.exists(sched.TIMINGS), reason="no measured timing set in the package")
def test_trained_network_gains_over_the_heuristic(engine):
    """Trained on the GPU from the committed autotuner timings (80 %), the MLP's
    BF16 choices on the held-out 20 % have lower regret than the shape
    heuristic (the method without it) and stay within 5 % of the autotuner."""
    d = np.load(sched.TIMINGS)
    shapes, dens, T = d["shapes"], d["density"], d["ms"]
    F = sched.raw_features(shapes[:, 0], shapes[:, 1], shapes[:, 2], shapes[:, 3], dens)
    cut = int(0.8 * len(F))
    mlp = sched.MLP(engine, seed=5)
    mlp.fit(F[:cut], T[:cut], epochs=150, batch=256, lr=2e-3)
    r_mlp = sched.regret(T[cut:], mlp.choose(F[cut:]))
    r_heur = sched.regret(T[cut:], sched.heuristic_choice(F[cut:]))
    assert r_mlp < r_heur
    assert r_mlp <= 0.05


@pytest.mark.skipif(not os.path.exists(sched.RANK_TIMINGS), reason="no measured rank timing set in the package")
def test_trained_rank_network_gains_over_the_rank_rule(engine):
    """The rank rounds' planner: trained on the GPU from the committed marginal
    rank timings (hme_autotune_batch_rank, 80 %), its BF16 choices on the
    held-out 20 % have lower regret than the rank rounds' batch rule (the method
    without it) and stay within 5 % of the autotuner."""
    d = np.load(sched.RANK_TIMINGS)
    shapes, dens, T = d["shapes"], d["density"], d["ms"]
    F = sched.raw_features(shapes[:, 0], shapes[:, 1], shapes[:, 2], shapes[:, 3], dens)
    cut = int(0.8 * len(F))
    mlp = sched.MLP(engine, seed=5)
    mlp.fit(F[:cut], T[:cut], epochs=300, batch=256, lr=2e-3)
    r_mlp = sched.regret(T[cut:], mlp.choose(F[cut:]))
    r_rule = sched.regret(T[cut:], sched.rank_rule(shapes[cut:, 1]))
    assert r_mlp < r_rule
    assert r_mlp <= 0.05


def test_plan_with_fallback_records_the_autotuners_choice(engine):
    """Where the network is not confident -- here a network whose outputs are all
    equal, so every class is a tie -- the exhaustive autotuner's best replaces
    the network's choice, once per shape class, in the returned plan and in the
    engine's plan (hme_sched_plan_set), which policy 1 then follows; the rank is
    unchanged.  The autotuner is a stand-in that prefers schedule 2."""
    import torch

    mlp = sched.MLP(engine, seed=1)
    mlp.set_params(np.zeros(mlp.n_params, np.float32))
    p, m, n, r = 2147483629, 200, 300, 120
    shapes = np.array([[65521, 48, 48, 48], [p, m, n, r], [p, m, n, r]], np.uint32)
    calls = []

    def tuner(pp, mm, nn, kk, dd):
        calls.append((int(pp), int(mm)))
        return np.array([3.0, 2.0, 1.0, 4.0])

    v, nfb = sched.plan_with_fallback(mlp, engine, shapes, rank=True, autotune_fn=tuner)
    assert nfb == 2 and len(calls) == 2 and list(v) == [2, 2, 2]
    L = _lib.lib()
    bad = np.array([4], np.int32)
    assert L.hme_sched_plan_set(engine._h, 1, 1, shapes[:1].ctypes.data_as(_lib.u32p),
                                bad.ctypes.data_as(C.POINTER(C.c_int))) == _lib.HME_EINVAL
    rng = np.random.default_rng(9)
    A = rng.integers(0, p, (m, r), dtype=np.uint64).astype(np.uint32)
    B = rng.integers(0, p, (r, n), dtype=np.uint64).astype(np.uint32)
    jobs = [{"p": p, "A": _dev(A), "B": _dev(B), "C": torch.zeros((m, n), dtype=torch.int32, device="cuda")}]
    try:
        _lib.check(L.hme_ctx_set_sched_policy(engine._h, 1))
        engine.set_timing(True)
        engine.timing_reset()
        ranks = engine.batch_gemm_rank_dev(jobs)
        _, simt_launches = engine.kernel_time("batch_simt_update")
    finally:
        engine.set_timing(False)
        _lib.check(L.hme_ctx_set_sched_policy(engine._h, 0))
    assert simt_launches > 0  # schedule 2: the CUDA-core update
    assert list(ranks) == [r]
