"""The learned scheduler's host side: features, the MLP handle, timing
collection with the exhaustive autotuner, training, planning and regret.

A schedule is a GEMM variant (hme_gemm_u32_dev_variant: 0 limb tcgen05 wide
tiles, 1 limb tcgen05 half-width tiles, 2 CUDA-core 32 x 32, 3 CUDA-core
64 x 64), and for a batched job's rank rounds a rank schedule (0 / 1 the
grouped tcgen05 limb GEMM as the trailing update, 2 / 3 the CUDA-core update;
0 / 2 finish a job in one last panel of up to 128 columns, 1 / 3 take 32-column
rounds to the end), each picked by its own network of the same shape, trained
on its own autotuner's timings.  Every variant computes the same residues (and
ranks), so neither the MLP nor the autotuner can change a value -- only the
time.  The MLP (5 -> 3 x 64 -> 4,
hand-written CUDA kernels: FP32 training, BF16 inference) predicts each
variant's normalised log-time from (log2 m, log2 n, log2 k, log2 p, density);
the exhaustive autotuner (hme_autotune_gemm) times all variants, supplies the
training data, judges the MLP's regret, and is its fallback where the network
is not confident (plan_with_fallback).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import check

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
WEIGHTS = os.path.join(DATA, "sched_mlp.npz")
TIMINGS = os.path.join(DATA, "sched_timings.npz")
# the batched stream's planner: trained on per-job times inside batches (hme_autotune_batch)
BATCH_WEIGHTS = os.path.join(DATA, "sched_batch_mlp.npz")
BATCH_TIMINGS = os.path.join(DATA, "sched_batch_timings.npz")
# the rank rounds' planner: trained on per-job marginal rank times beside an anchor job (hme_autotune_batch_rank)
RANK_WEIGHTS = os.path.join(DATA, "sched_rank_mlp.npz")
RANK_TIMINGS = os.path.join(DATA, "sched_rank_timings.npz")
BATCH_RULE = -1
N_VARIANTS = 4
VARIANT_NAMES = ("tensor-wide", "tensor-narrow", "simt-32", "simt-64")
# schedules of a batched job's rank rounds: trailing-update variant, widest last panel (columns)
N_RANK_VARIANTS = 4
RANK_VARIANT_NAMES = ("tensor/last-128", "tensor/last-32", "simt/last-128", "simt/last-32")


def rank_rule(m) -> np.ndarray:
    """The rank rounds' batch rule (the method without the planner): schedule 0
    (tensor-core update, one last panel of up to 128 columns) for jobs of at most
    128 rows, else 1 (32-column rounds to the end); as jobs.cu rank_rule."""
    return np.where(np.asarray(m) <= 128, 0, 1).astype(np.int32)

_fp = C.POINTER(C.c_float)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def raw_features(p, m, n, k, density) -> np.ndarray:
    p, m, n, k, d = (np.asarray(x, dtype=np.float64) for x in (p, m, n, k, density))
    return np.stack([np.log2(m), np.log2(n), np.log2(k), np.log2(p), d], axis=-1)


class MLP:
    """One scheduler network on an Engine's device (libhme hme_mlp)."""

    def __init__(self, engine, seed: int = 1):
        self._lib = _lib.lib()
        self.engine = engine
        h = C.c_void_p()
        check(self._lib.hme_mlp_create(engine._h, seed, C.byref(h)))
        self._h = h
        self.n_params = int(self._lib.hme_mlp_param_count())
        self.x_mean = np.zeros(5, np.float32)
        self.x_std = np.ones(5, np.float32)
        self.y_mean = 0.0
        self.y_std = 1.0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hme_mlp_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters --------------------------------------------------------------
    def get_params(self) -> np.ndarray:
        w = np.zeros(self.n_params, np.float32)
        check(self._lib.hme_mlp_get_params(self._h, w.ctypes.data_as(_fp)))
        return w

    def set_params(self, w) -> None:
        w = _f32(w)
        assert w.size == self.n_params
        check(self._lib.hme_mlp_set_params(self._h, w.ctypes.data_as(_fp)))

    def save(self, path: str = WEIGHTS) -> None:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.get_params(), x_mean=self.x_mean, x_std=self.x_std,
                 y_mean=np.float32(self.y_mean), y_std=np.float32(self.y_std))

    def load(self, path: str = WEIGHTS) -> None:
        d = np.load(path)
        self.set_params(d["params"])
        self.x_mean, self.x_std = d["x_mean"].astype(np.float32), d["x_std"].astype(np.float32)
        self.y_mean, self.y_std = float(d["y_mean"]), float(d["y_std"])

    # ---- raw kernels on normalised data ------------------------------------------------
    def loss_grad(self, X, Y):
        X, Y = _f32(X), _f32(Y)
        loss = C.c_float()
        g = np.zeros(self.n_params, np.float32)
        check(self._lib.hme_mlp_loss_grad(self._h, X.shape[0], X.ctypes.data_as(_fp), Y.ctypes.data_as(_fp),
                                          C.byref(loss), g.ctypes.data_as(_fp)))
        return loss.value, g

    def train_normalised(self, X, Y, epochs=200, batch=256, lr=2e-3, seed=7) -> float:
        X, Y = _f32(X), _f32(Y)
        loss = C.c_float()
        check(self._lib.hme_mlp_train(self._h, X.shape[0], X.ctypes.data_as(_fp), Y.ctypes.data_as(_fp), epochs,
                                      batch, lr, seed, C.byref(loss)))
        return loss.value

    def predict_normalised(self, X) -> np.ndarray:
        X = _f32(X)
        Y = np.zeros((X.shape[0], N_VARIANTS), np.float32)
        check(self._lib.hme_mlp_predict_bf16(self._h, X.shape[0], X.ctypes.data_as(_fp), Y.ctypes.data_as(_fp)))
        return Y

    # ---- on raw features / measured times ------------------------------------------------
    def fit(self, F, T, **kw) -> float:
        """Train on raw features F (n x 5) and measured times T (n x 4, ms)."""
        F = np.asarray(F, np.float64)
        self.x_mean = F.mean(0).astype(np.float32)
        self.x_std = np.maximum(F.std(0), 1e-3).astype(np.float32)
        L = np.log(np.maximum(np.asarray(T, np.float64), 1e-6))
        self.y_mean, self.y_std = float(L.mean()), float(max(L.std(), 1e-3))
        return self.train_normalised((F - self.x_mean) / self.x_std, (L - self.y_mean) / self.y_std, **kw)

    def choose(self, F) -> np.ndarray:
        F = np.asarray(F, np.float64)
        return np.argmin(self.predict_normalised((F - self.x_mean) / self.x_std), axis=1)

    def norm(self) -> np.ndarray:
        return np.concatenate([self.x_mean, self.x_std]).astype(np.float32)

    def plan(self, shapes, density=None) -> np.ndarray:
        """hme_sched_plan: BF16 inference + arg-min for rows (p, m, n, k); records the
        decisions in the engine's learned plan (policy 1)."""
        S = np.ascontiguousarray(shapes, dtype=np.uint32)
        n = S.shape[0]
        d = _f32(np.ones(n) if density is None else density)
        v = np.zeros(max(1, n), np.int32)
        nm = self.norm()
        check(self._lib.hme_sched_plan(self.engine._h, self._h, n, S.ctypes.data_as(_lib.u32p),
                                       d.ctypes.data_as(_fp), nm.ctypes.data_as(_fp),
                                       v.ctypes.data_as(C.POINTER(C.c_int))))
        return v[:n]

    def predict_ms(self, F) -> np.ndarray:
        """Predicted per-variant times (ms) for raw features F (n x 5), BF16 inference."""
        F = np.asarray(F, np.float64)
        Y = self.predict_normalised((F - self.x_mean) / self.x_std).astype(np.float64)
        return np.exp(Y * self.y_std + self.y_mean)

    def plan_rank(self, shapes, density=None) -> np.ndarray:
        """hme_sched_plan_rank: the same for the rank rounds' schedules (a network
        trained on hme_autotune_batch_rank timings); records the decisions in the
        engine's rank plan (policy 1)."""
        S = np.ascontiguousarray(shapes, dtype=np.uint32)
        n = S.shape[0]
        d = _f32(np.ones(n) if density is None else density)
        v = np.zeros(max(1, n), np.int32)
        nm = self.norm()
        check(self._lib.hme_sched_plan_rank(self.engine._h, self._h, n, S.ctypes.data_as(_lib.u32p),
                                            d.ctypes.data_as(_fp), nm.ctypes.data_as(_fp),
                                            v.ctypes.data_as(C.POINTER(C.c_int))))
        return v[:n]


def fallback_classes(shapes, predicted_ms, margin: float):
    """The shape classes where a network is not confident: its best predicted
    time is within `margin` (relative) of its second best for some job of the
    class.  Returns {class: index of its first such job}."""
    T = np.sort(np.asarray(predicted_ms, np.float64), axis=1)
    unsure = T[:, 1] <= T[:, 0] * (1.0 + margin)
    first = {}
    for t in np.nonzero(unsure)[0]:
        first.setdefault(shape_class(*shapes[t]), int(t))
    return first


def plan_with_fallback(mlp, engine, shapes, density=None, rank: bool = False, margin: float = 0.03,
                       autotune_fn=None):
    """Per-job schedules from a planner network with the exhaustive autotuner as
    its fallback: the network plans every job (hme_sched_plan / _plan_rank), and
    in each shape class where it is not confident (fallback_classes) the
    autotuner times every variant once and its best replaces the network's
    choice, in the returned array and in the engine's plan (hme_sched_plan_set),
    so policy 1 follows it too.  Returns (variants, classes that fell back)."""
    S = np.ascontiguousarray(shapes, dtype=np.uint32)
    n = S.shape[0]
    d = np.ones(n) if density is None else np.asarray(density, np.float64)
    v = (mlp.plan_rank if rank else mlp.plan)(S, d).copy()
    if n == 0:
        return v, 0
    first = fallback_classes(S, mlp.predict_ms(raw_features(S[:, 0], S[:, 1], S[:, 2], S[:, 3], d)), margin)
    if rank:  # jobs of more than 1024 rows take the single-matrix elimination: no rank schedule to choose
        first = {key: t for key, t in first.items() if S[t, 1] <= 1024}
    if not first:
        return v, 0
    if autotune_fn is None:
        autotune_fn = ((lambda p, m, nn, k, dd: autotune_batch_rank(engine, p, m, nn, k, dd)) if rank
                       else (lambda p, m, nn, k, dd: autotune_batch(engine, p, m, nn, k)))
    best = {key: int(np.argmin(autotune_fn(*S[t], d[t]))) for key, t in first.items()}
    for t in range(n):
        b = best.get(shape_class(*S[t]))
        if b is not None:
            v[t] = b
    rows = np.ascontiguousarray([S[t] for t in first.values()], dtype=np.uint32)
    vals = np.ascontiguousarray([best[key] for key in first], dtype=np.int32)
    check(_lib.lib().hme_sched_plan_set(engine._h, 1 if rank else 0, len(vals), rows.ctypes.data_as(_lib.u32p),
                                        vals.ctypes.data_as(C.POINTER(C.c_int))))
    return v, len(first)


def heuristic_choice(F, num_sms: int = 148) -> np.ndarray:
    """The method without the MLP: always the tensor-core GEMM, wide tiles unless
    fewer than 3/4 of the SMs would get one (the engine's shape heuristic)."""
    F = np.asarray(F, np.float64)
    m, n, p = 2.0 ** F[:, 0], 2.0 ** F[:, 1], 2.0 ** F[:, 3]
    L = np.where(p <= 256, 1, np.where(p <= 65536, 2, np.where(p <= 2 ** 24, 3, 4)))
    bn = np.maximum(256 // L, 64)
    tiles = np.ceil(m / 128) * np.ceil(n / bn)
    return np.where(4 * tiles < 3 * num_sms, 1, 0)


def regret(T, choice) -> float:
    """Mean relative excess time of the chosen variants over the best measured ones."""
    T = np.asarray(T, np.float64)
    best = T.min(1)
    got = T[np.arange(T.shape[0]), np.asarray(choice)]
    return float(np.mean((got - best) / best))


def sample_shapes(n: int, seed: int = 11):
    """Seeded GEMM shapes drawn from the configurations' mix: config-4 jobs
    (squares 16..1024, both moduli, dense or banded), config-2/3 trailing
    updates (m, n 64..2048, k in {32, 64, 128}, p = 2^31 - 19, 2^16, 3^10) and
    config-1 products (128..2048 cubes at 65521).  Rows (p, m, n, k), density."""
    rng = np.random.default_rng(seed)
    kind = rng.integers(0, 3, n)
    P = np.zeros(n, np.int64)
    S = np.zeros((n, 3), np.int64)
    dens = np.ones(n)
    for i in range(n):
        if kind[i] == 0:
            s = int(np.rint(16 * 64 ** rng.random()))
            P[i] = (65521, 2147483629)[rng.integers(0, 2)]
            S[i] = (s, s, s)
            dens[i] = (1.0, 0.05)[rng.integers(0, 2)]
        elif kind[i] == 1:
            P[i] = (2147483629, 65536, 59049)[rng.integers(0, 3)]
            S[i] = (int(64 * 32 ** rng.random()), int(64 * 32 ** rng.random()), (32, 64, 128)[rng.integers(0, 3)])
        else:
            s = int(128 * 16 ** rng.random())
            P[i] = 65521
            S[i] = (s, s, s)
    return np.column_stack([P, S]).astype(np.uint32), dens


def autotune(engine, p, m, n, k, reps: int = 3) -> np.ndarray:
    ms = np.zeros(N_VARIANTS, np.float32)
    check(_lib.lib().hme_autotune_gemm(engine._h, int(p), int(m), int(n), int(k), reps, ms.ctypes.data_as(_fp)))
    return ms


def batch_count(m, n, k, work: float = 2.0 ** 27, cap: int = 256) -> int:
    """Jobs of one shape timed together by the batch autotuner: about `work`
    multiply-adds per batch, at least one job, at most `cap`."""
    return int(max(1, min(cap, work // max(1, int(m) * int(n) * int(k)))))


def autotune_batch(engine, p, m, n, k, count=None, reps: int = 3) -> np.ndarray:
    """Per-job device time (ms) of every GEMM variant inside a batch of `count`
    jobs of this shape (hme_autotune_batch)."""
    ms = np.zeros(N_VARIANTS, np.float32)
    c = batch_count(m, n, k) if count is None else int(count)
    check(_lib.lib().hme_autotune_batch(engine._h, int(p), int(m), int(n), int(k), c, reps, ms.ctypes.data_as(_fp)))
    return ms


def rank_batch_count(m, n, k, work: float = 2.0 ** 27, cap: int = 256) -> int:
    """Jobs of one shape whose ranks the rank autotuner times together: about
    `work` elimination multiply-adds (m n min(m, n, k)) per batch, 1 .. `cap`."""
    r = max(1, min(int(m), int(n), int(k)))
    return int(max(1, min(cap, work // max(1, int(m) * int(n) * r))))


def autotune_batch_rank(engine, p, m, n, k, density=1.0, count=None, reps: int = 3) -> np.ndarray:
    """Per-job marginal device time (ms) of every rank schedule: what `count`
    products of this shape add to a batch whose rounds run anyway (beside a
    dense 1024 x 1024 anchor job; hme_autotune_batch_rank)."""
    ms = np.zeros(N_RANK_VARIANTS, np.float32)
    c = rank_batch_count(m, n, k) if count is None else int(count)
    check(_lib.lib().hme_autotune_batch_rank(engine._h, int(p), int(m), int(n), int(k), float(density), c, reps,
                                             ms.ctypes.data_as(_fp)))
    return ms


def shape_class(p, m, n, k) -> tuple:
    """Quarter-octave class of a product's shape and its limb count (the key of
    the engine's plan table, sched.cu shape_key)."""
    q = lambda x: int(np.rint(4.0 * np.log2(max(1, int(x)))))  # noqa: E731
    p = int(p)
    L = 1 if p <= 256 else 2 if p <= 65536 else 3 if p <= (1 << 24) else 4
    return (q(m), q(n), q(k), L)


def sample_stream_shapes(n: int, seed: int = 11):
    """Seeded job shapes of the batched stream's mix (stream.MixedStream): config-4
    jobs (squares 16..1024, p in {65521, 2^31 - 19}, dense or banded), config-2
    products (s x r times r x s, s 64..1024, r = s - s // 20, p = 2^31 - 19) and
    config-1 cubes (128..1024 at 65521).  Rows (p, m, n, k), density."""
    rng = np.random.default_rng(seed)
    kind = rng.choice(3, size=n, p=[0.6, 0.25, 0.15])
    P = np.zeros(n, np.int64)
    S = np.zeros((n, 3), np.int64)
    dens = np.ones(n)
    for i in range(n):
        if kind[i] == 0:
            s = int(np.rint(16 * 64 ** rng.random()))
            P[i] = (65521, 2147483629)[rng.integers(0, 2)]
            S[i] = (s, s, s)
            dens[i] = (1.0, 0.05)[rng.integers(0, 2)]
        elif kind[i] == 1:
            s = int(np.rint(64 * 16 ** rng.random()))
            P[i] = 2147483629
            S[i] = (s, s, s - s // 20)
        else:
            s = int(np.rint(128 * 8 ** rng.random()))
            P[i] = 65521
            S[i] = (s, s, s)
    return np.column_stack([P, S]).astype(np.uint32), dens


def collect_batch(engine, n: int, seed: int = 11, reps: int = 3, budget_s=None):
    """Time every variant inside batches on n seeded stream shapes: (shapes, density, per-job ms)."""
    shapes, dens = sample_stream_shapes(n, seed)
    return _timed_rows(shapes, dens, N_VARIANTS, lambda i: autotune_batch(engine, *shapes[i], reps=reps), budget_s)


def _timed_rows(shapes, dens, nv, time_row, budget_s):
    """Time rows in order until all are done or `budget_s` seconds have passed:
    (shapes, density, T) of the rows timed."""
    import time

    T = np.zeros((len(shapes), nv), np.float32)
    t0, done = time.perf_counter(), 0
    for i in range(len(shapes)):
        T[i] = time_row(i)
        done = i + 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    return shapes[:done], dens[:done], T[:done]


def collect_batch_rank(engine, n: int, seed: int = 11, reps: int = 3, budget_s=None):
    """Time every rank schedule inside batches on n seeded stream shapes: (shapes, density, per-job ms)."""
    shapes, dens = sample_stream_shapes(n, seed)
    return _timed_rows(shapes, dens, N_RANK_VARIANTS,
                       lambda i: autotune_batch_rank(engine, *shapes[i], dens[i], reps=reps), budget_s)


def collect(engine, n: int, seed: int = 11, reps: int = 3, budget_s=None):
    """Time every variant on n seeded shapes: (shapes, density, times ms)."""
    shapes, dens = sample_shapes(n, seed)
    return _timed_rows(shapes, dens, N_VARIANTS, lambda i: autotune(engine, *shapes[i], reps), budget_s)
