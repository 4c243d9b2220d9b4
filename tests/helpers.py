"""Shared helpers for the parity tests."""
import json

import numpy as np

from tests.conftest import GOLDEN


def load_golden(name):
    G = np.load(GOLDEN / f"{name}.npz")
    return G, json.loads(str(G["meta"]))


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
