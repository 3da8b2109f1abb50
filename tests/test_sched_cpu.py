"""CPU tests of the scheduler's oracle and host logic: the numpy MLP reference's
gradient against central finite differences, the bf16 rounding, and the
regret / heuristic bookkeeping."""
import numpy as np

from oracle import mlp_ref as R
from hacs_b200 import sched


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(0, 0.3, R.N_PARAMS)
    X = rng.normal(0, 1, (17, R.N_IN))
    Y = rng.normal(0, 1, (17, R.N_OUT))
    loss, g = R.loss_grad(w, X, Y)
    idx = rng.choice(R.N_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(R.N_PARAMS)
        e[i] = h
        fd = (R.loss_grad(w + e, X, Y)[0] - R.loss_grad(w - e, X, Y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 3.14159265, -2.5e-3, 65504.0], np.float32)
    r = R.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie at 1 + 2^-8 rounds to even
    assert r[2] == np.float32(1.0078125)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


def test_regret_and_heuristic():
    T = np.array([[1.0, 2.0, 3.0, 4.0], [5.0, 1.0, 2.0, 2.0]])
    assert sched.regret(T, [0, 1]) == 0.0
    assert abs(sched.regret(T, [1, 0]) - 2.5) < 1e-12
    F = sched.raw_features([65521, 65521], [8192, 16], [8192, 16], [8192, 16], [1, 1])
    assert list(sched.heuristic_choice(F)) == [0, 1]


def test_shape_sampler_is_seeded():
    a, da = sched.sample_shapes(50, 3)
    b, db = sched.sample_shapes(50, 3)
    assert np.array_equal(a, b) and np.array_equal(da, db)
    assert a[:, 1:].min() >= 16 and a[:, 1:].max() <= 4096


def test_rank_batch_count_and_timing_budget():
    """The rank autotuner's batch sizes (about 2^27 elimination multiply-adds per
    batch, 1 .. 256 jobs) and the collection loop's time budget (rows are timed
    in order; the rows timed so far are kept when the budget runs out)."""
    assert sched.rank_batch_count(16, 16, 16) == 256
    assert sched.rank_batch_count(1024, 1024, 1024) == 1
    assert sched.rank_batch_count(200, 300, 20) == 2 ** 27 // (200 * 300 * 20)
    shapes, dens = sched.sample_stream_shapes(7, seed=3)
    calls = []

    def row(i):
        calls.append(i)
        return np.full(sched.N_RANK_VARIANTS, i + 1.0)

    s, d, T = sched._timed_rows(shapes, dens, sched.N_RANK_VARIANTS, row, None)
    assert calls == list(range(7)) and T.shape == (7, 4) and np.array_equal(s, shapes)
    calls.clear()
    s, d, T = sched._timed_rows(shapes, dens, sched.N_RANK_VARIANTS, row, -1.0)  # budget spent after row 0
    assert calls == [0] and len(s) == len(d) == len(T) == 1 and T[0, 0] == 1.0


def test_fallback_classes_pick_unconfident_shapes():
    """A shape class falls back to the exhaustive autotuner when, for some job of
    the class, the network's best predicted time is within the margin of its
    second best; one job per class is timed."""
    shapes = np.array([[65521, 100, 100, 100], [65521, 101, 101, 101],  # one class (quarter octaves)
                       [65521, 500, 500, 500], [2147483629, 500, 500, 500]], np.uint32)
    T = np.array([[1.00, 1.01, 2.0, 3.0],   # within 3 %: unsure
                  [1.00, 1.50, 2.0, 3.0],   # same class, confident
                  [1.00, 1.20, 2.0, 3.0],   # confident
                  [2.00, 2.05, 2.0, 9.0]])  # a tie: unsure
    first = sched.fallback_classes(shapes, T, 0.03)
    assert sched.shape_class(*shapes[0]) == sched.shape_class(*shapes[1])
    assert first == {sched.shape_class(*shapes[0]): 0, sched.shape_class(*shapes[3]): 3}
    assert sched.fallback_classes(shapes, T, 0.0) == {sched.shape_class(*shapes[3]): 3}
