"""CPU reference of the learned warm-start network (test infrastructure only).

Restates, in numpy, the forward pass and the gradient of the mean squared
error that libwpsph's tensor-core kernels compute, with the same BF16 rounding
points: standardised inputs, weights, hidden activations and the
back-propagated layer-2/layer-1 deltas are rounded to bfloat16 (round to
nearest even) before each product; sums are taken in float64 here (the GPU
accumulates in FP32, which is the difference the tests tolerate).

Blob layout (include/wpsph.h): mu[10], sd[10], t_scale, then W1[10][64],
b1[64], W2[64][64], b2[64], w3[64], b3 with W[in][out].
"""

from __future__ import annotations

import numpy as np

NF, NH = 10, 64
OFF_MU, OFF_SD, OFF_TS = 0, 10, 20
P0 = 21
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


def forward(blob, feat):
    w = unpack(blob)
    inv_sd = (np.float32(1.0) / w["sd"]).astype(np.float32)
    x = ((np.asarray(feat, np.float32) - w["mu"]) * inv_sd).astype(np.float32)
    xb = bf16(x).astype(np.float64)
    W1, W2, w3 = (bf16(w[k]).astype(np.float64) for k in ("W1", "W2", "w3"))
    z1 = xb @ W1 + w["b1"]
    h1 = bf16(np.maximum(z1, 0).astype(np.float32)).astype(np.float64)
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
