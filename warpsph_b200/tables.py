"""Cubic-spline kernel tables (sph_funcs.py:47-86).

W(q) = sigma (6 (q^3 - q^2) + 1) for q <= 1/2, 2 sigma (1 - q)^3 for 1/2 < q < 1,
0 beyond; the gradient table stores -(dW/dr)/r, i.e. (12 - 18 q) sigma / h^2 and
6 sigma (1 - q)^2 / (h r).  Samples are at linspace(0, h, S), evaluated in FP64
and stored as float32.  The arithmetic sequence matches the reference's numpy
code operation for operation, which makes the float32 tables bit-identical.
"""

from __future__ import annotations

import numpy as np

from .params import SolverParams


def kernel_tables(p: SolverParams) -> tuple[np.ndarray, np.ndarray]:
    h = p.h
    sigma = p.sigma
    h_inv = 1.0 / h
    h_inv2 = 1.0 / (h * h)
    r_w = np.linspace(0, h, p.w_table_size, dtype=np.float64)
    r_g = np.linspace(0, h, p.g_table_size, dtype=np.float64)
    q_w = r_w * h_inv
    q_g = r_g * h_inv

    w = np.zeros_like(r_w)
    inner = q_w <= 0.5
    outer = (q_w > 0.5) & (q_w < 1.0)
    w[inner] = (6.0 * (q_w[inner] ** 3 - q_w[inner] ** 2) + 1.0) * sigma
    w[outer] = 2.0 * np.power(1.0 - q_w[outer], 3) * sigma

    g = np.zeros_like(r_g)
    nonzero = r_g > 1e-10
    inner = nonzero & (q_g <= 0.5)
    outer = nonzero & (q_g > 0.5) & (q_g < 1.0)
    g[inner] = (12.0 - 18.0 * q_g[inner]) * sigma * h_inv2
    g[outer] = 6.0 * np.power(1.0 - q_g[outer], 2) * sigma * h_inv / r_g[outer]
    return w.astype(np.float32), g.astype(np.float32)
