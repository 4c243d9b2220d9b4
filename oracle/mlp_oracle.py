"""CPU reference of the learned warm-start network (test infrastructure only).

Restates, in numpy, the forward pass and the gradient of the mean squared
error that libwpsph's tensor-core kernels compute, with the same BF16 rounding
points: standardised inputs, weights, hidden activations and the
back-propagated layer-2/layer-1 deltas are rounded to bfloat16 (round to
nearest even) before each product; sums are taken in float64 here (the
training kernels accumulate in FP32, which is the difference the tests
tolerate), or, for the step's tensor-core inference, as that kernel
accumulates (``forward(..., tc=True)``).

Blob layout (include/wpsph.h): mu[11], sd[11], t_scale, then W1[11][64],
b1[64], W2[64][64], b2[64], w3[64], b3 with W[in][out].
"""

from __future__ import annotations

import numpy as np

NF, NH = 11, 64
OFF_MU, OFF_SD, OFF_TS = 0, NF, 2 * NF
P0 = 2 * NF + 1
SIZES = [("W1", (NF, NH)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("w3", (NH,)), ("b3", (1,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)
BLOB = P0 + NPARAMS


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(blob):
    blob = np.asarray(blob, dtype=np.float32)
    out, off = {}, P0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = blob[off:off + k].reshape(shape)
        off += k
    out["mu"] = blob[OFF_MU:OFF_MU + NF]
    out["sd"] = blob[OFF_SD:OFF_SD + NF]
    out["t_scale"] = float(blob[OFF_TS])
    return out


def trunc32(a) -> np.ndarray:
    """float64 values rounded toward zero to float32."""
    a = np.asarray(a, np.float64)
    b = a.astype(np.float32)
    over = np.abs(b.astype(np.float64)) > np.abs(a)
    b[over] = np.nextafter(b[over], np.float32(0))
    return b


def forward(blob, feat, tc=False):
    """Forward pass.  tc=False: the products summed exactly (float64).
    tc=True: as the step's tensor-core inference kernel accumulates, which
    this restatement matches by taking each layer's exact dot product rounded
    toward zero to float32 before the float32 bias add (measured: with the
    float64 sums instead, single hidden units land on the other side of a
    BF16 rounding boundary and the output moves by ~5e-4)."""
    w = unpack(blob)
    inv_sd = (np.float32(1.0) / w["sd"]).astype(np.float32)
    x = ((np.asarray(feat, np.float32) - w["mu"]) * inv_sd).astype(np.float32)
    xb = bf16(x).astype(np.float64)
    W1, W2, w3 = (bf16(w[k]).astype(np.float64) for k in ("W1", "W2", "w3"))
    if tc:
        z1 = (trunc32(xb @ W1) + w["b1"]).astype(np.float64)
    else:
        z1 = xb @ W1 + w["b1"]
    h1 = bf16(np.maximum(z1, 0).astype(np.float32)).astype(np.float64)
    if tc:
        z2 = (trunc32(h1 @ W2) + w["b2"]).astype(np.float64)
    else:
        z2 = h1 @ W2 + w["b2"]
    h2 = bf16(np.maximum(z2, 0).astype(np.float32)).astype(np.float64)
    y = h2 @ w3 + w["b3"][0]
    return dict(xb=xb, z1=z1, h1=h1, z2=z2, h2=h2, y=y, W2=W2, w3=w3)


def loss_and_grad(blob, feat, target):
    """Mean squared error of y against target / t_scale and its gradient in
    blob parameter order (W1, b1, W2, b2, w3, b3)."""
    w = unpack(blob)
    f = forward(blob, feat)
    n = len(f["y"])
    tn = np.asarray(target, np.float32) * np.float32(1.0 / w["t_scale"])
    e = f["y"] - tn
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    dw3 = f["h2"].T @ dy
    db3 = np.array([dy.sum()])
    dz2 = np.outer(dy, f["w3"]) * (f["z2"] > 0)
    db2 = dz2.sum(0)
    dz2b = bf16(dz2.astype(np.float32)).astype(np.float64)
    dh1 = dz2b @ f["W2"].T
    dz1 = dh1 * (f["z1"] > 0)
    db1 = dz1.sum(0)
    dz1b = bf16(dz1.astype(np.float32)).astype(np.float64)
    dW2 = f["h1"].T @ dz2b
    dW1 = f["xb"].T @ dz1b
    grad = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dw3, db3])
    return loss, grad, f["y"]


# ------------------------------------------------------------ warm-start inputs and start

def _f32(x):
    return np.float32(x)


def column_top_depth(x, grid):
    """Input 10's depth: per fluid particle, the highest fluid y of its
    neighbour-grid column (x, z) minus its own y, clamped at 0.  ``grid`` is
    sph_get_grid's output (origin, 1 / cell (y, z), 1 / cell along x, cells
    per axis); cell coordinates are float32 floor((x - origin) / cell),
    clamped to the grid, as the library computes them."""
    x = np.asarray(x, np.float32).reshape(-1, 3)
    ox, oy, oz, inv, inv_x = (np.float32(g) for g in grid[:5])
    nx, ny, nz = (int(g) for g in grid[5:8])
    cx = np.clip(np.floor((x[:, 0] - ox) * inv_x), 0, nx - 1).astype(np.int64)
    cz = np.clip(np.floor((x[:, 2] - oz) * inv), 0, nz - 1).astype(np.int64)
    col = cz * nx + cx
    top = np.full(nx * nz, -np.inf, np.float32)
    np.maximum.at(top, col, x[:, 1])
    return np.maximum(top[col] - x[:, 1], np.float32(0))


def warm_start_features(step, x, p_prev, bx, psi, w_table, consts, dt, grid):
    """The network's 11 inputs per fluid particle, restated in float32 numpy
    from an oracle step's exported terms (oracle.step(..., export=True)) and
    the step's input positions x.

    The inputs are built from the reference's own per-particle quantities:
    rho_adv (predict_rho_adv, IISPH.py:281-329), a_ii (compute_term_a,
    IISPH.py:385-428), d_ii (compute_term_d, IISPH.py:332-382), the
    neighbour counts (IISPH.py:52-163) and the boundary share of the density
    (compute_density, IISPH.py:177-214).  grad rho = m sum_j gradW_ij +
    sum_b psi_b gradW_ib is recovered from d_ii = -grad rho dt^2 / rho^2.
    ``consts``: dict with rho0, gravity, h, omega, inv_small, fluid_mass and
    w_size (the W table's samples); ``grid``: sph_get_grid's output (input 10,
    column_top_depth)."""
    rho = np.asarray(step["rho"], np.float32)
    rho_adv = np.asarray(step["rho_adv"], np.float32)
    aii = np.asarray(step["a_ii"], np.float32)
    dii = np.asarray(step["d_ii"], np.float32)
    n = len(rho)
    rho0, grav, h = _f32(consts["rho0"]), _f32(consts["gravity"]), _f32(consts["h"])
    omega, inv_small, m = _f32(consts["omega"]), _f32(consts["inv_small"]), _f32(consts["fluid_mass"])
    dt = _f32(dt)
    dt2 = dt * dt
    rr = rho * rho
    inv_rho0 = _f32(1.0) / rho0
    p_ref = _f32(1.0) / (rho0 * grav * h)
    h2 = h * h
    h4 = h2 * h2
    aa = aii.copy()
    small = (aa > -inv_small) & (aa < inv_small)
    aa[small] = np.where(aa[small] < 0, _f32(-1.0), _f32(1.0)) * inv_small
    p1 = np.maximum((rho0 - rho_adv) * omega / aa, _f32(0.0))
    grad = (-dii) * (rr / dt2)[:, None]
    # boundary share of the density: sum_b psi_b W(|x_i - x_b|) over each fluid-boundary list
    off = np.asarray(step["fb_off"], np.int64)
    idx = np.asarray(step["fb_idx"], np.int64)
    xi = np.repeat(np.asarray(x, np.float32).reshape(-1, 3), np.diff(off), axis=0)
    d = xi - np.asarray(bx, np.float32)[idx]
    r = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(np.float32)
    S = int(consts["w_size"])
    T = np.asarray(w_table, np.float32)
    f = r * (_f32(S - 1) * (_f32(1.0) / h))
    lo = np.minimum(f.astype(np.int64), S - 2)
    a = f - lo.astype(np.float32)
    w = (_f32(1.0) - a) * T[lo] + a * T[lo + 1]
    w[r >= h] = 0
    sWb = np.zeros(n, np.float64)
    np.add.at(sWb, np.repeat(np.arange(n), np.diff(off)), (w * np.asarray(psi, np.float32)[idx]).astype(np.float64))
    F = np.zeros((n, NF), np.float32)
    F[:, 0] = rho_adv * inv_rho0 - _f32(1.0)
    F[:, 1] = (rho_adv - rho) * inv_rho0
    F[:, 2] = aii * rr / (dt2 * m * m) * h4 * h4
    F[:, 3] = np.arcsinh(np.asarray(p_prev, np.float32) * p_ref)
    F[:, 4] = np.diff(np.asarray(step["ff_off"], np.int64)).astype(np.float32)
    F[:, 5] = sWb.astype(np.float32) * inv_rho0
    F[:, 6] = np.sqrt((grad * grad).sum(1)).astype(np.float32) * h * inv_rho0
    F[:, 7] = np.arcsinh(p1 * p_ref)
    F[:, 8] = grad[:, 1] * h * inv_rho0
    F[:, 9] = np.diff(off).astype(np.float32)
    F[:, 10] = np.arcsinh(column_top_depth(x, grid) / h)
    return F


def solve_start(blob, feat, consts, max_rise=0.5):
    """The pressure a learned-start step's Jacobi solve begins from
    (replacing init_pressure, IISPH.py:166-174): the network's correction y
    on top of the base u = max(input 3, input 10) (the previous step's
    pressure and the column's hydrostatic pressure, carried in float32), its
    rise bounded by max_rise, clamped at 0 and mapped back:
    p = sinh(max(u + min(y t_scale, max_rise), 0)) rho0 g h."""
    feat = np.asarray(feat, np.float32)
    y = forward(blob, feat, tc=True)["y"].astype(np.float32)
    ts = np.float32(unpack(blob)["t_scale"])
    u = np.maximum(feat[:, 3], feat[:, 10])
    p_unit = np.float32(float(consts["rho0"]) * float(consts["gravity"]) * float(consts["h"]))
    t = np.maximum(u + np.minimum(y * ts, np.float32(max_rise)), np.float32(0.0))
    return (np.sinh(t.astype(np.float32)) * p_unit).astype(np.float32)
