"""Shared helpers for the parity tests."""
import json

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
