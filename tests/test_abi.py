"""The C ABI library loads without a GPU and exports every symbol declared in
include/wpsph.h; struct layouts agree with the ctypes mirror; host-only entry
points (defaults, tables, ABI info) work on the CPU."""
import ctypes
import re

import numpy as np

from tests.conftest import ROOT
from tests.helpers import load_golden


def declared_functions():
    text = (ROOT / "include" / "wpsph.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sph_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from warpsph_b200 import _lib
    from warpsph_b200.build import build

    build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes binding covers exactly the declared set
    assert sorted(_lib.SIGNATURES) == names


def test_struct_layouts_match():
    from warpsph_b200 import _lib

    L = _lib.load()
    info = np.zeros(4, np.int32)
    assert L.sph_abi_info(_lib.ptr(info), 4) == 0
    assert info[0] == 1
    assert info[1] == ctypes.sizeof(_lib.SphParams)
    assert info[2] == ctypes.sizeof(_lib.SphStepStats)


def test_defaults_match_reference_constants():
    from warpsph_b200 import _lib
    from warpsph_b200.params import SolverParams

    L = _lib.load()
    c = _lib.SphParams()
    assert L.sph_params_default(ctypes.byref(c)) == 0
    py = SolverParams().to_c()
    for name, _ in _lib.SphParams._fields_:
        a, b = getattr(c, name), getattr(py, name)
        if isinstance(a, (int, float)):
            assert a == b, name
    import wp_sph.main as m

    assert c.h == m.SMOOTHING_LENGTH and c.fluid_mass == m.FLUID_MASS and c.sigma == m.SIGMA
    assert c.dt_max == m.TIME_STEP_MAX


def test_library_tables_match_reference():
    """The tables libwpsph builds by itself are the reference's (golden) tables."""
    from warpsph_b200 import _lib
    from warpsph_b200.params import SolverParams
    from warpsph_b200.tables import kernel_tables

    L = _lib.load()
    for name in ("ref_lattice", "dam_jitter"):
        G, meta = load_golden(name)
        p = SolverParams(diameter=meta["diameter"], w_table_size=meta["w_size"], g_table_size=meta["g_size"])
        w = np.zeros(p.w_table_size, np.float32)
        g = np.zeros(p.g_table_size, np.float32)
        assert L.sph_build_tables(ctypes.byref(p.to_c()), _lib.ptr(w), _lib.ptr(g)) == 0
        assert np.array_equal(w, G["W_table"])
        assert np.array_equal(g, G["grad_W_table"])
        pw, pg = kernel_tables(p)
        assert np.array_equal(pw, G["W_table"]) and np.array_equal(pg, G["grad_W_table"])


def test_create_fails_loudly_without_gpu():
    """No CUDA device here: sph_create must return an error, never fall back."""
    import torch

    from warpsph_b200 import _lib

    if torch.cuda.is_available():
        return
    L = _lib.load()
    ctx = ctypes.c_void_p()
    p = _lib.SphParams()
    L.sph_params_default(ctypes.byref(p))
    assert L.sph_create(ctypes.byref(p), ctypes.byref(ctx)) != 0
    assert not ctx.value
