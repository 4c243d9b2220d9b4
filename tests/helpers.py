"""Shared helpers for the parity tests."""
import json
import math

import numpy as np

from tests.conftest import GOLDEN


def load_golden(name):
    G = np.load(GOLDEN / f"{name}.npz")
    return G, json.loads(str(G["meta"]))


def golden_oracle_params(oracle, meta):
    """Oracle constants of a golden scene (main.py:25-61 as make_golden patched them)."""
    return oracle.reference_params(diameter=meta["diameter"], gravity=meta["gravity"], w_size=meta["w_size"],
                                   g_size=meta["g_size"], vis_mu_scale=meta.get("vis_mu", 0.0) / meta["rho0"])


def golden_solver_params(meta, **kw):
    """SolverParams of a golden scene."""
    from warpsph_b200.params import SolverParams

    return SolverParams(diameter=meta["diameter"], gravity=meta["gravity"], w_table_size=meta["w_size"],
                        g_table_size=meta["g_size"], vis_mu_scale=meta.get("vis_mu", 0.0) / meta["rho0"], **kw)


def normrel(a, b):
    """max |a - b| / max |b|: the norm-wise relative error used by the parity bar."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.max(np.abs(b)) if b.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(a))) if a.size else 0.0
    return float(np.max(np.abs(a - b)) / scale)


def csr_equal(off_a, idx_a, off_b, idx_b):
    return np.array_equal(np.asarray(off_a), np.asarray(off_b)) and np.array_equal(
        np.asarray(idx_a), np.asarray(idx_b))


# ------------------------------------------------------------------ per-element parity
#
# Per-element relative error: |a_i - b_i| / max(|b_i|, floor) for scalars and
# |a_i - b_i|_2 / max(|b_i|_2, floor) for vectors (one value per particle).
# The floor is the quantity's own physical scale below which a relative error
# stops meaning anything (a near-zero pressure at the free surface, the
# cancellation residual d_ii of an interior particle whose neighbours surround
# it); elements above the floor are compared purely relatively.

def gradient_unit(h):
    """|grad W| of the cubic spline at r = h/2 (one particle spacing):
    the inner branch (12 - 18 q) sigma / h^2 times r at q = 1/2 is 1.5 sigma / h,
    sigma = 8 / (pi h^3) (sph_funcs.py:79-82)."""
    return 12.0 / (math.pi * h ** 4)


def parity_floors(params, dt):
    """Floors per quantity, from the scene's physical scales:
      rho, rho_adv  1 % of rho0 (never binds: an isolated particle has rho0/pi)
      p             hydrostatic pressure of one particle layer, rho0 g d
      Ap            the solve's tolerance in density units, eta rho0
      d_ii          one neighbour's term at the spacing, dt^2 m |gradW(d)| / rho0^2
      s             that term times the pressure floor
      a_ii          one neighbour's term of a_ii, (dt m |gradW(d)| / rho0)^2
      v             the velocity gravity adds in one step, g dt
      x             the particle spacing d (x errors are displacements)"""
    d = params.diameter
    h = 2 * d
    rho0 = params.rho0
    m = rho0 * d ** 3
    g1 = gradient_unit(h)
    p_floor = rho0 * params.gravity * d
    dterm = dt * dt * m * g1 / rho0 ** 2
    return {"rho": 0.01 * rho0, "rho_adv": 0.01 * rho0, "p": p_floor, "Ap": params.eta * rho0,
            "d_ii": dterm, "s": dterm * p_floor, "a_ii": (dt * m * g1 / rho0) ** 2,
            "v": params.gravity * dt, "v_adv": params.gravity * dt, "x": d}


def elemrel(a, b, floor, x_like=False):
    """Per-element relative errors (a vector of one value per particle).
    x_like: the error is the displacement |a - b| over the floor alone."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.ndim == 2:
        diff = np.linalg.norm(a - b, axis=1)
        mag = np.linalg.norm(b, axis=1)
    else:
        diff = np.abs(a - b)
        mag = np.abs(b)
    if x_like:
        return diff / floor
    return diff / np.maximum(mag, floor)


def elemstats(a, b, floor, x_like=False):
    """(max, 99.9th percentile) of the per-element relative error."""
    e = elemrel(a, b, floor, x_like)
    if e.size == 0:
        return 0.0, 0.0
    return float(e.max()), float(np.percentile(e, 99.9))


# The relaxed-Jacobi outputs (p, s, Ap) of an FP32 evaluation move by ~5e-4 of
# a single particle's value with the summation order alone (the update divides
# the small residual rho0 - rho_adv - Ap by a_ii); a result counts as matching
# when it is within 1e-4 of the reference or no further from the FP64 oracle
# than NOISE times the reference's own FP32 result is.
NOISE = 4.0


def jacobi_output_ok(got, ref, truth, floor, bar=1e-4):
    """(ok, detail) for a Jacobi output compared per element."""
    g_ref = elemstats(got, ref, floor)
    if g_ref[0] < bar:
        return True, {"vs_ref": g_ref}
    g_truth = elemstats(got, truth, floor)
    r_truth = elemstats(ref, truth, floor)
    return g_truth[0] <= NOISE * r_truth[0], {"vs_ref": g_ref, "vs_fp64": g_truth, "ref_vs_fp64": r_truth}
