"""Collect autotuner timings on this GPU and train the scheduler MLP.

    python -m hacs_b200.sched_train [--shapes 20000] [--reps 3] [--epochs 300] [--batch]

Times every GEMM variant on `--shapes` seeded shapes from the configurations'
mix with the exhaustive autotuner (hme_autotune_gemm), trains the MLP on the
GPU (hme_mlp_train: the library's FP32 forward / backward / Adam kernels) on
80 % of them, reports the BF16-inference regret against the autotuner's best on
the other 20 % next to the shape heuristic's, and writes
hacs_b200/data/sched_timings.npz and hacs_b200/data/sched_mlp.npz.

--batch trains the batched stream's planner instead: every variant is timed
per job inside a batch of same-shape jobs (hme_autotune_batch, the cost a job
adds to a batched call), written to sched_batch_timings.npz and
sched_batch_mlp.npz; the method without the network is the batch rule.

--rank trains the planner of the batched rank rounds: every rank schedule
(trailing-update variant x widest last panel) is timed per job inside a
batch of same-shape products (hme_autotune_batch_rank), written to
sched_rank_timings.npz and sched_rank_mlp.npz; the method without the network
is the rank rounds' batch rule (sched.rank_rule).
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import hacs_b200  # noqa: E402
from hacs_b200 import sched  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--shapes", type=int, default=20000)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--reuse", action="store_true", help="train on the existing timing file")
    ap.add_argument("--batch", action="store_true", help="the batched stream's planner (per-job times in batches)")
    ap.add_argument("--rank", action="store_true", help="the rank rounds' planner (per-job rank times in batches)")
    ap.add_argument("--budget-s", type=float, default=None,
                    help="stop timing shapes after this many seconds and train on the shapes timed so far")
    ap.add_argument("--out-dir", default=None, help="write the timing and weight files here (default: the package)")
    args = ap.parse_args()
    if args.rank:
        timings, weights = sched.RANK_TIMINGS, sched.RANK_WEIGHTS
    else:
        timings = sched.BATCH_TIMINGS if args.batch else sched.TIMINGS
        weights = sched.BATCH_WEIGHTS if args.batch else sched.WEIGHTS
    nv = sched.N_RANK_VARIANTS if args.rank else sched.N_VARIANTS
    if args.out_dir:
        os.makedirs(args.out_dir, exist_ok=True)
        timings = os.path.join(args.out_dir, os.path.basename(timings))
        weights = os.path.join(args.out_dir, os.path.basename(weights))
    eng = hacs_b200.Engine(0)
    if args.reuse and os.path.exists(timings):
        d = np.load(timings)
        shapes, dens, T = d["shapes"], d["density"], d["ms"]
    else:
        t0 = time.time()
        collect = sched.collect_batch_rank if args.rank else sched.collect_batch if args.batch else sched.collect
        shapes, dens, T = collect(eng, args.shapes, args.seed, args.reps, budget_s=args.budget_s)
        print(f"timed {len(shapes)} shapes x {nv} variants in {time.time() - t0:.1f} s", flush=True)
        os.makedirs(os.path.dirname(timings), exist_ok=True)
        np.savez_compressed(timings, shapes=shapes, density=dens, ms=T)
    F = sched.raw_features(shapes[:, 0], shapes[:, 1], shapes[:, 2], shapes[:, 3], dens)
    n = len(F)
    cut = int(0.8 * n)
    mlp = sched.MLP(eng, seed=5)
    t0 = time.time()
    loss = mlp.fit(F[:cut], T[:cut], epochs=args.epochs, batch=256, lr=2e-3)
    tt = time.time() - t0
    mlp.save(weights)
    ch = mlp.choose(F[cut:])
    rule = sched.rank_rule(shapes[cut:, 1]) if args.rank else None
    rep = {"train_shapes": cut, "test_shapes": n - cut, "train_loss": loss, "train_s": tt,
           "regret_mlp": sched.regret(T[cut:], ch),
           "regret_heuristic": (sched.regret(T[cut:], rule) if args.rank else None if args.batch
                                else sched.regret(T[cut:], sched.heuristic_choice(F[cut:]))),
           # variant 0: wide tensor-core tiles (GEMM planners); the batch rule (rank planner)
           "regret_variant0": sched.regret(T[cut:], np.zeros(n - cut, int)),
           "variant_share_best": np.bincount(T[cut:].argmin(1), minlength=nv).tolist(),
           "variant_share_mlp": np.bincount(ch, minlength=nv).tolist()}
    print(json.dumps(rep), flush=True)


if __name__ == "__main__":
    main()
