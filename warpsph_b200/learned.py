"""Learned pressure warm start: data collection, training and storage.

The network (11 -> 64 -> 64 -> 1, BF16 tensor cores) is trained on the
solver's own converged pressures: every step of a set of dam-break scenes
exports each particle's 11 inputs and asinh(p / (rho0 g h)) of its converged
pressure (sph_get_features), a sample of them forms the training set, and
sph_mlp_train fits the network on the GPU (Adam, MSE).  The network is
residual: it predicts the change of asinh(p / (rho0 g h)) from a base, the
larger of the previous step's value (input 3) and the hydrostatic pressure of
the fluid column above the particle (input 10), which the inference kernel
adds back in float32, so the network's BF16 arithmetic only touches the
correction.  At run time SPH_WARM_MLP starts the relaxed Jacobi solve from the
prediction; the solve's stopping rule is unchanged.

Inputs (computed in the neighbour build, all dimensionless):
 0 rho_adv / rho0 - 1            predicted density deviation
 1 (rho_adv - rho) / rho0        velocity divergence over the step
 2 a_ii rho^2 h^8 / (m dt)^2     diagonal of the pressure system
 3 asinh(p_prev / (rho0 g h))    previous step's pressure
 4 fluid neighbour count
 5 sum_b psi_b W_ib / rho0       boundary share of the density
 6 |grad rho| h / rho0
 7 asinh(p_1 / (rho0 g h))       first Jacobi iterate from p = 0
 8 (grad rho)_y h / rho0         density gradient along gravity
 9 boundary neighbour count
10 asinh(depth / h)              hydrostatic pressure of the fluid column above:
                                 depth below the highest fluid particle of the
                                 particle's neighbour-grid column (x, z)
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _lib

NF, NH = _lib.SPH_MLP_FEATURES, 64
BLOB = _lib.SPH_MLP_BLOB
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "warm_start_mlp.npz"


def init_blob(feat: np.ndarray, target: np.ndarray, seed: int = 0) -> np.ndarray:
    """Input standardisation from the data, output unit = target std, He-initialised weights."""
    rng = np.random.default_rng(seed)
    mu = feat.mean(0).astype(np.float32)
    sd = feat.std(0).astype(np.float32)
    sd = np.maximum(sd, 1e-6 * (np.abs(mu) + 1.0)).astype(np.float32)
    t_scale = np.float32(max(float(target.std()), 1e-6))
    w1 = rng.normal(0, np.sqrt(2.0 / NF), (NF, NH))
    w2 = rng.normal(0, np.sqrt(2.0 / NH), (NH, NH))
    w3 = rng.normal(0, np.sqrt(1.0 / NH), (NH,))
    parts = [mu, sd, [t_scale], w1.ravel(), np.zeros(NH), w2.ravel(), np.zeros(NH), w3, [float(target.mean()) / t_scale]]
    blob = np.concatenate([np.asarray(p, np.float64).ravel() for p in parts]).astype(np.float32)
    assert blob.size == BLOB
    return blob


PREV, HYDRO = 3, 10  # inputs whose larger value is carried around the network


def base(feat) -> np.ndarray:
    """The residual's base: max(asinh(p_prev / (rho0 g h)), asinh(depth / h))."""
    f = np.asarray(feat, np.float32)
    return np.maximum(f[:, PREV], f[:, HYDRO])


def residual_target(feat, target) -> np.ndarray:
    """What the network regresses: the target minus the base."""
    return (np.asarray(target, np.float32) - base(feat)).astype(np.float32)


def train(feat, target, epochs=20, batch=4096, lr=1e-3, seed=0, device=0, blob=None):
    """Fit the network on the GPU to (feat, target), target = asinh(p / (rho0 g h))
    of the converged pressure; returns (blob, per-epoch loss)."""
    feat = np.ascontiguousarray(feat, np.float32)
    target = np.ascontiguousarray(residual_target(feat, target), np.float32)
    blob = init_blob(feat, target, seed) if blob is None else np.array(blob, np.float32)
    cfg = _lib.SphMlpTrainConfig(epochs=epochs, batch=batch, lr=lr, beta1=0.9, beta2=0.999, eps=1e-8,
                                 seed=seed, device=device)
    losses = np.zeros(max(epochs, 1), np.float32)
    rc = _lib.load().sph_mlp_train(ctypes.byref(cfg), _lib.ptr(feat), _lib.ptr(target), len(target),
                                   _lib.ptr(blob), _lib.ptr(losses))
    _lib.check(None, rc)
    return blob, losses[:epochs]


def predict(blob, feat, device=0) -> np.ndarray:
    """Predicted asinh(p / (rho0 g h)) before the clamp at 0: the base plus
    the network's correction, whose rise is bounded by SPH_MLP_MAX_RISE."""
    feat = np.ascontiguousarray(feat, np.float32)
    y = evaluate(blob, feat, device=device)
    return base(feat) + np.minimum(y * np.float32(blob[2 * NF]), np.float32(_lib.SPH_MLP_MAX_RISE))


def evaluate(blob, feat, target=None, device=0):
    """Network outputs (units of t_scale) and, with a target (already residual),
    (loss, gradient) of the mean squared error."""
    feat = np.ascontiguousarray(feat, np.float32)
    blob = np.ascontiguousarray(blob, np.float32)
    pred = np.zeros(len(feat), np.float32)
    grad = None
    t = None
    if target is not None:
        t = np.ascontiguousarray(target, np.float32)
        grad = np.zeros(_lib.SPH_MLP_PARAMS + 1, np.float32)
    rc = _lib.load().sph_mlp_eval(_lib.ptr(blob), _lib.ptr(feat), _lib.ptr(t), len(feat), device,
                                  _lib.ptr(pred), _lib.ptr(grad))
    _lib.check(None, rc)
    if grad is None:
        return pred
    return pred, float(grad[-1]), grad[:-1]


def collect(scenes, steps, per_step, params_for, seed=0, warm="zero", skip=0, skip_capped=True,
            early_steps=0, early_boost=1):
    """Run each scene for ``steps`` steps, sampling ``per_step`` (input, target)
    pairs per step after the first ``skip`` steps, ``early_boost`` times as
    many in the first ``early_steps`` (the start-up transient, a small share
    of the steps but where a start saves the most iterations).  With
    ``skip_capped``, steps whose solve stopped at the iteration cap are left
    out: their pressure is not a solution of the step's system.
    ``params_for(scene)`` gives the SolverParams."""
    from .solver import IISPH

    rng = np.random.default_rng(seed)
    feats, targets = [], []
    for sc in scenes:
        sol = IISPH(stage_path=None, params=params_for(sc).replace(warm_start=warm), scene=sc)
        _lib.check(sol._ctx, sol._lib.sph_set_record_features(sol._ctx, 1))
        n = sc.n
        f = np.zeros((n, NF), np.float32)
        t = np.zeros(n, np.float32)
        for k in range(steps):
            sol.step()
            if k < skip or (skip_capped and sol.last_stats["flags"] & _lib.SPH_F_NOT_CONVERGED):
                continue
            _lib.check(sol._ctx, sol._lib.sph_get_features(sol._ctx, _lib.ptr(f), _lib.ptr(t)))
            want = per_step * (early_boost if k < early_steps else 1)
            pick = rng.choice(n, size=min(want, n), replace=False)
            feats.append(f[pick].copy())
            targets.append(t[pick].copy())
        sol.close()
    return np.concatenate(feats), np.concatenate(targets)


def weighted_resample(feat, target, alpha, seed=0):
    """Resample (feat, target) with replacement, pair k drawn with weight
    1 + alpha * max(target_k, 0): the mean-squared loss then weighs the
    pressurised interior, whose error sets how many Jacobi iterations a step
    needs, above the free surface and splashes."""
    t = np.asarray(target, np.float32)
    w = 1.0 + alpha * np.maximum(t.astype(np.float64), 0.0)
    pick = np.random.default_rng(seed).choice(len(t), size=len(t), replace=True, p=w / w.sum())
    return np.ascontiguousarray(np.asarray(feat, np.float32)[pick]), np.ascontiguousarray(t[pick])


def save(path, blob, **meta):
    np.savez_compressed(path, blob=np.asarray(blob, np.float32), **meta)


def load_blob(path=DEFAULT_WEIGHTS) -> np.ndarray:
    return np.load(path)["blob"].astype(np.float32)
