"""ctypes wrapper around the CPU oracle (``liboracle_sph.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference leg, never by the product package.

``kernel_tables`` restates the reference's table construction
(wp_sph/solver/sph_funcs.py:47-86) in numpy; ``reference_params`` restates the
constants of wp_sph/main.py:25-61.  ``step`` runs one reference time step
(IISPH.py:1002-1371) in FP32 (mirror) or FP64 (truth).
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_sph.so"


class OracleParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in (
        "h", "h_inv", "rho0", "gravity", "omega", "eta", "inv_small", "vis_mu",
        "fluid_mass", "dt_max", "cfl_len")] + [(k, ctypes.c_int) for k in (
            "w_size", "g_size", "max_loop", "min_loop", "fixed_iters", "err_fp32_seq",
            "nthreads", "warm_start")]


class OracleStep(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64), ("nb", ctypes.c_int64),
        ("x", ctypes.c_void_p), ("v", ctypes.c_void_p), ("p", ctypes.c_void_p),
        ("bx", ctypes.c_void_p), ("bv", ctypes.c_void_p), ("psi", ctypes.c_void_p),
        ("w_table", ctypes.c_void_p), ("g_table", ctypes.c_void_p),
        ("dt", ctypes.c_double), ("inv_dt", ctypes.c_double),
        ("rho", ctypes.c_void_p), ("v_adv", ctypes.c_void_p), ("rho_adv", ctypes.c_void_p),
        ("d_ii", ctypes.c_void_p), ("a_ii", ctypes.c_void_p), ("s", ctypes.c_void_p),
        ("Ap", ctypes.c_void_p),
        ("ff_off", ctypes.c_void_p), ("ff_idx", ctypes.c_void_p), ("ff_cap", ctypes.c_int64),
        ("fb_off", ctypes.c_void_p), ("fb_idx", ctypes.c_void_p), ("fb_cap", ctypes.c_int64),
        ("iterations", ctypes.c_int), ("status", ctypes.c_int),
        ("avg_err", ctypes.c_double), ("v_max", ctypes.c_double),
        ("dt_next", ctypes.c_double), ("inv_dt_next", ctypes.c_double),
        ("n_ff_pairs", ctypes.c_int64), ("n_fb_pairs", ctypes.c_int64),
    ]


_LIB = None


def build():
    """Compile liboracle_sph.so with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER(OracleParams)
        L.oracle_step_f32.argtypes = [P, ctypes.POINTER(OracleStep)]
        L.oracle_step_f64.argtypes = [P, ctypes.POINTER(OracleStep)]
        for name in ("oracle_psi_f32", "oracle_psi_f64"):
            getattr(L, name).argtypes = [P, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_neighbors_f32.argtypes = [P, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                           ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
        L.oracle_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# --------------------------------------------------------------- constants

def reference_params(diameter=0.05, gravity=9.8, w_size=8192, g_size=65536, rho0=1.0e3,
                     omega=0.5, eta=1.0e-3, inv_small=1.0e-6, vis_mu_scale=0.0, **_):
    """Derived constants as wp_sph/main.py:25-61 and sph_funcs.py:6-9 compute them."""
    h = 2 * diameter
    return dict(
        diameter=diameter, h=h, h_inv=1.0 / h, rho0=rho0, gravity=gravity, omega=omega, eta=eta,
        inv_small=inv_small, vis_mu=vis_mu_scale * rho0, fluid_mass=rho0 * diameter**3,
        dt_max=5e-2 * diameter, cfl_len=0.4 * diameter, sigma=8 / (math.pi * h**3),
        w_size=w_size, g_size=g_size)


def kernel_tables(params: dict, dtype=np.float32):
    """Cubic-spline W and (dW/dr)/r tables as sph_funcs.py:47-86 build them (FP64,
    then cast).  The arithmetic sequence is kept identical so the float32 tables
    are bit-identical to the reference's."""
    h = params["h"]
    sigma = params["sigma"]
    h_inv = 1.0 / h
    h_inv2 = 1.0 / (h * h)
    r_w = np.linspace(0, h, params["w_size"], dtype=np.float64)
    r_g = np.linspace(0, h, params["g_size"], dtype=np.float64)
    q_w = r_w * h_inv
    q_g = r_g * h_inv
    w = np.zeros_like(r_w)
    lo = q_w <= 0.5
    hi = (q_w > 0.5) & (q_w < 1.0)
    w[lo] = (6.0 * (q_w[lo] ** 3 - q_w[lo] ** 2) + 1.0) * sigma
    w[hi] = 2.0 * np.power(1.0 - q_w[hi], 3) * sigma
    g = np.zeros_like(r_g)
    nz = r_g > 1e-10
    lo = nz & (q_g <= 0.5)
    hi = nz & (q_g > 0.5) & (q_g < 1.0)
    g[lo] = (12.0 - 18.0 * q_g[lo]) * sigma * h_inv2
    g[hi] = 6.0 * np.power(1.0 - q_g[hi], 2) * sigma * h_inv / r_g[hi]
    return w.astype(dtype), g.astype(dtype)


def _c_params(params: dict, fixed_iters=-1, err_fp32_seq=False, nthreads=0, warm_start=0,
              max_loop=100, min_loop=2) -> OracleParams:
    return OracleParams(
        h=params["h"], h_inv=params["h_inv"], rho0=params["rho0"], gravity=params["gravity"],
        omega=params["omega"], eta=params["eta"], inv_small=params["inv_small"],
        vis_mu=params["vis_mu"], fluid_mass=params["fluid_mass"], dt_max=params["dt_max"],
        cfl_len=params["cfl_len"], w_size=params["w_size"], g_size=params["g_size"],
        max_loop=max_loop, min_loop=min_loop, fixed_iters=fixed_iters,
        err_fp32_seq=int(err_fp32_seq), nthreads=nthreads or max_threads(), warm_start=warm_start)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def boundary_psi(params: dict, bx, tables=None, precision="f32", nthreads=0):
    dt = np.float32 if precision == "f32" else np.float64
    w, _ = tables if tables is not None else kernel_tables(params, dt)
    bx = np.ascontiguousarray(bx, dtype=dt)
    w = np.ascontiguousarray(w, dtype=dt)
    out = np.zeros(len(bx), dtype=dt)
    P = _c_params(params, nthreads=nthreads)
    fn = lib().oracle_psi_f32 if precision == "f32" else lib().oracle_psi_f64
    rc = fn(ctypes.byref(P), len(bx), _ptr(bx), _ptr(w), _ptr(out))
    assert rc == 0
    return out


def neighbors(params: dict, xq, xs, same: bool, cap_per_query=128, nthreads=0):
    """Exact FP32 neighbour sets {j : |xq_i - xs_j| < h} as CSR (offsets, ids)."""
    xq = np.ascontiguousarray(xq, dtype=np.float32)
    xs = np.ascontiguousarray(xs, dtype=np.float32)
    off = np.zeros(len(xq) + 1, dtype=np.int64)
    cap = max(1, len(xq) * cap_per_query)
    idx = np.zeros(cap, dtype=np.int32)
    P = _c_params(params, nthreads=nthreads)
    rc = lib().oracle_neighbors_f32(ctypes.byref(P), len(xq), _ptr(xq), len(xs), _ptr(xs),
                                    int(same), _ptr(off), _ptr(idx), cap)
    assert rc == 0, "neighbour capacity exceeded"
    return off, idx[: off[-1]].copy()


def step(params: dict, x, v, bx, bv, psi, dt, inv_dt=None, p=None, tables=None,
         precision="f32", fixed_iters=-1, err_fp32_seq=False, export=True,
         nthreads=0, warm_start=0, cap_per_particle=128):
    """One reference IISPH step.  Returns a dict of the new state and, with
    ``export``, every intermediate quantity and the neighbour sets."""
    dt_np = np.float32 if precision == "f32" else np.float64
    n, nb = len(x), len(bx)
    w, g = tables if tables is not None else kernel_tables(params, dt_np)
    arrs = dict(
        x=np.array(x, dtype=dt_np, order="C").reshape(n, 3),
        v=np.array(v, dtype=dt_np, order="C").reshape(n, 3),
        p=(np.zeros(n, dt_np) if p is None else np.array(p, dtype=dt_np)),
        bx=np.ascontiguousarray(bx, dtype=dt_np).reshape(nb, 3),
        bv=(np.zeros((nb, 3), dt_np) if bv is None else np.ascontiguousarray(bv, dtype=dt_np)),
        psi=np.ascontiguousarray(psi, dtype=dt_np),
        w=np.ascontiguousarray(w, dtype=dt_np), g=np.ascontiguousarray(g, dtype=dt_np))
    S = OracleStep(n=n, nb=nb, x=_ptr(arrs["x"]), v=_ptr(arrs["v"]), p=_ptr(arrs["p"]),
                   bx=_ptr(arrs["bx"]), bv=_ptr(arrs["bv"]), psi=_ptr(arrs["psi"]),
                   w_table=_ptr(arrs["w"]), g_table=_ptr(arrs["g"]), dt=float(dt),
                   inv_dt=float(1.0 / dt if inv_dt is None else inv_dt))
    out = {}
    if export:
        for k, shape in (("rho", (n,)), ("v_adv", (n, 3)), ("rho_adv", (n,)), ("d_ii", (n, 3)),
                         ("a_ii", (n,)), ("s", (n, 3)), ("Ap", (n,))):
            out[k] = np.zeros(shape, dt_np)
            setattr(S, k, _ptr(out[k]))
        cap = max(1, n * cap_per_particle)
        ff_off = np.zeros(n + 1, np.int64)
        fb_off = np.zeros(n + 1, np.int64)
        ff_idx = np.zeros(cap, np.int32)
        fb_idx = np.zeros(cap, np.int32)
        S.ff_off, S.ff_idx, S.ff_cap = _ptr(ff_off), _ptr(ff_idx), cap
        S.fb_off, S.fb_idx, S.fb_cap = _ptr(fb_off), _ptr(fb_idx), cap
    P = _c_params(params, fixed_iters=fixed_iters, err_fp32_seq=err_fp32_seq, nthreads=nthreads,
                  warm_start=warm_start)
    fn = lib().oracle_step_f32 if precision == "f32" else lib().oracle_step_f64
    rc = fn(ctypes.byref(P), ctypes.byref(S))
    assert rc == 0, f"oracle step failed ({rc})"
    if export:
        out["ff_off"], out["ff_idx"] = ff_off, ff_idx[: ff_off[-1]].copy()
        out["fb_off"], out["fb_idx"] = fb_off, fb_idx[: fb_off[-1]].copy()
    out.update(x=arrs["x"], v=arrs["v"], p=arrs["p"], iterations=S.iterations, avg_err=S.avg_err,
               v_max=S.v_max, dt_next=S.dt_next, inv_dt_next=S.inv_dt_next,
               n_ff_pairs=S.n_ff_pairs, n_fb_pairs=S.n_fb_pairs)
    return out
