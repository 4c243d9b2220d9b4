"""Train the shipped learned warm-start network (GPU).

    python -m warpsph_b200.train_warm_start [--pairs 2000000] [--steps 400] [--epochs 20] [--rounds 2]

Data: the solver's own converged pressures on the 64 batched dam-break scenes
(`scenes.batched_scenes`, 0.01 m spacing, dt 5e-4, 1024-sample tables,
g = 9.81), `--steps` steps each, sampled evenly to `--pairs` pairs after each
scene's first `--skip` steps (default none: the start-up transient is in the
data), leaving out steps whose solve stopped at the iteration cap (their
pressure solves nothing).  Training: Adam, lr 1e-3, MSE, on the GPU with
libwpsph's own kernels.

The first fit uses data from the reference's own runs (p = 0 start).  Each of
`--rounds` further rounds collects with the previous network as the warm
start, the states the shipped solver visits (its first steps converge, where
the p = 0 runs hit the cap), and fits a fresh network to that data resampled
with weight 1 + alpha * max(target, 0) (`learned.weighted_resample`).
Output: warpsph_b200/data/warm_start_mlp.npz.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import learned
from .params import SolverParams
from .scenes import batched_scenes


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=2_000_000)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=str(learned.DEFAULT_WEIGHTS))
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--skip", type=int, default=0, help="start-up steps of each scene left out of the data")
    ap.add_argument("--rounds", type=int, default=2, help="on-policy rounds after the first fit")
    ap.add_argument("--alpha", type=float, default=1.0, help="resampling weight 1 + alpha * max(target, 0)")
    ap.add_argument("--early-steps", type=int, default=0, help="steps of each scene sampled early-boost times as densely")
    ap.add_argument("--early-boost", type=int, default=1)
    a = ap.parse_args()
    scenes = batched_scenes(count=a.scenes)
    per_step = max(1, a.pairs // (a.scenes * max(1, a.steps - a.skip)))
    t0 = time.time()
    params = SolverParams(diameter=0.01, gravity=9.81, w_table_size=1024, g_table_size=1024)
    early = dict(early_steps=a.early_steps, early_boost=a.early_boost)
    feat, target = learned.collect(scenes, a.steps, per_step, lambda sc: params, seed=a.seed, warm="zero",
                                   skip=a.skip, **early)
    t_collect = time.time() - t0
    t1 = time.time()
    blob, losses = learned.train(feat, target, epochs=a.epochs, lr=a.lr, seed=a.seed)
    t_train = time.time() - t1
    for r in range(1, a.rounds + 1):
        t0 = time.time()
        policy = params.replace(extra={"mlp_blob": blob})
        feat, target = learned.collect(scenes, a.steps, per_step, lambda sc: policy, seed=a.seed + r, warm="mlp",
                                       skip=a.skip, **early)
        feat, target = learned.weighted_resample(feat, target, a.alpha, seed=a.seed + r)
        t_collect += time.time() - t0
        t1 = time.time()
        blob, losses = learned.train(feat, target, epochs=a.epochs, lr=a.lr, seed=a.seed)
        t_train += time.time() - t1
    meta = dict(pairs=len(target), scenes=a.scenes, steps=a.steps, skip=a.skip, early_steps=a.early_steps,
                early_boost=a.early_boost, epochs=a.epochs, lr=a.lr,
                rounds=a.rounds, alpha=a.alpha, losses=losses.tolist(), collect_s=t_collect, train_s=t_train)
    learned.save(a.out, blob, meta=json.dumps(meta))
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
