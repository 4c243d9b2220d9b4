"""ctypes binding of libwpsph.so (the C ABI declared in include/wpsph.h).

The CUDA library is the only compute path: if it is missing or no CUDA device
is usable, every entry point raises instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libwpsph.so"

SPH_OK = 0
SPH_E_INVALID = -1
SPH_E_CUDA = -2
SPH_E_CAPACITY = -3
SPH_E_NONFINITE = -4
SPH_E_TIMEOUT = -5
SPH_E_NOMEM = -6
SPH_E_TOO_LARGE = -7
SPH_NOALLOC_MAX_BOUNDARY = 262144

SPH_F_FF_OVERFLOW = 0x1
SPH_F_FB_OVERFLOW = 0x2
SPH_F_NONFINITE = 0x4
SPH_F_TIMEOUT = 0x8
SPH_F_NOT_CONVERGED = 0x10

SPH_WARM_ZERO = 0
SPH_WARM_HALF = 1
SPH_WARM_MLP = 2

_ERRNAMES = {
    SPH_E_INVALID: "SPH_E_INVALID", SPH_E_CUDA: "SPH_E_CUDA", SPH_E_CAPACITY: "SPH_E_CAPACITY",
    SPH_E_NONFINITE: "SPH_E_NONFINITE", SPH_E_TIMEOUT: "SPH_E_TIMEOUT", SPH_E_NOMEM: "SPH_E_NOMEM",
    SPH_E_TOO_LARGE: "SPH_E_TOO_LARGE",
}


class SphError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class SphParams(ctypes.Structure):
    _fields_ = [
        ("spacing", ctypes.c_double), ("h", ctypes.c_double), ("rho0", ctypes.c_double),
        ("gravity", ctypes.c_double), ("omega", ctypes.c_double), ("eta", ctypes.c_double),
        ("inv_small", ctypes.c_double), ("vis_mu", ctypes.c_double), ("fluid_mass", ctypes.c_double),
        ("sigma", ctypes.c_double), ("dt_max", ctypes.c_double), ("cfl_len", ctypes.c_double),
        ("dt0", ctypes.c_double), ("domain_min", ctypes.c_double * 3), ("domain_max", ctypes.c_double * 3),
        ("w_table_size", ctypes.c_int32), ("g_table_size", ctypes.c_int32), ("min_iter", ctypes.c_int32),
        ("max_loop", ctypes.c_int32), ("fixed_iters", ctypes.c_int32), ("warm_start", ctypes.c_int32),
        ("max_ff", ctypes.c_int32), ("max_fb", ctypes.c_int32), ("keep_fb_lists", ctypes.c_int32),
        ("use_graph", ctypes.c_int32), ("device", ctypes.c_int32), ("block_size", ctypes.c_int32),
        ("timeout_ms", ctypes.c_int32), ("jacobi_block", ctypes.c_int32), ("jacobi_ppt", ctypes.c_int32),
        ("jacobi_unroll", ctypes.c_int32), ("move_boundary", ctypes.c_int32),
        ("warm_continue", ctypes.c_int32), ("plain_loads", ctypes.c_int32),
    ]


class SphMlpTrainConfig(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("seed", ctypes.c_uint32), ("device", ctypes.c_int32)]


SPH_MLP_FEATURES = 11
SPH_MLP_PARAMS = 4993
SPH_MLP_BLOB = 5016
SPH_MLP_MAX_RISE = 0.5


class SphSceneDesc(ctypes.Structure):
    _fields_ = [("x3", ctypes.c_void_p), ("v3", ctypes.c_void_p), ("n", ctypes.c_int64),
                ("xb3", ctypes.c_void_p), ("vb3", ctypes.c_void_p), ("nb", ctypes.c_int64),
                ("domain_min", ctypes.c_double * 3), ("domain_max", ctypes.c_double * 3)]


class SphStepStats(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32), ("flags", ctypes.c_int32), ("avg_err", ctypes.c_double),
        ("v_max", ctypes.c_double), ("dt", ctypes.c_double), ("dt_next", ctypes.c_double),
        ("sim_time", ctypes.c_double), ("n_ff_pairs", ctypes.c_int64), ("n_fb_pairs", ctypes.c_int64),
        ("max_ff_count", ctypes.c_int32), ("max_fb_count", ctypes.c_int32), ("step_index", ctypes.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.c_void_p
_F = ctypes.POINTER(ctypes.c_float)
# name: (restype, argtypes) — exactly the declarations of include/wpsph.h
SIGNATURES = {
    "sph_params_default": (ctypes.c_int, [ctypes.POINTER(SphParams)]),
    "sph_create": (ctypes.c_int, [ctypes.POINTER(SphParams), ctypes.POINTER(_P)]),
    "sph_destroy": (None, [_P]),
    "sph_last_error": (ctypes.c_char_p, [_P]),
    "sph_set_tables": (ctypes.c_int, [_P, _P, ctypes.c_int32, _P, ctypes.c_int32]),
    "sph_add_fluid": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64]),
    "sph_build_tables": (ctypes.c_int, [ctypes.POINTER(SphParams), _P, _P]),
    "sph_set_boundary": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64]),
    "sph_set_fluid": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64]),
    "sph_update_fluid": (ctypes.c_int, [_P, _P, _P, _P, ctypes.c_int64]),
    "sph_set_pressure": (ctypes.c_int, [_P, _P, ctypes.c_int64]),
    "sph_step": (ctypes.c_int, [_P, ctypes.POINTER(SphStepStats)]),
    "sph_steps": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(SphStepStats)]),
    "sph_get_stats_history": (ctypes.c_int, [_P, ctypes.POINTER(SphStepStats), ctypes.c_int32]),
    "sph_launch_steps": (ctypes.c_int, [_P, ctypes.c_int32]),
    "sph_launch_phase": (ctypes.c_int, [_P, ctypes.c_int32]),
    "sph_test_stall_barrier": (ctypes.c_int, [_P, ctypes.c_int32]),
    "sph_test_withhold_mma": (ctypes.c_int, [_P, ctypes.c_int32]),
    "sph_prepare": (ctypes.c_int, [_P]),
    "sph_neighbor_search": (ctypes.c_int, [_P]),
    "sph_get_fluid": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "sph_get_terms": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "sph_get_boundary": (ctypes.c_int, [_P, _P, _P]),
    "sph_get_neighbors": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P, _P, ctypes.c_int64]),
    "sph_get_stats": (ctypes.c_int, [_P, ctypes.POINTER(SphStepStats)]),
    "sph_set_dt": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double]),
    "sph_abi_info": (ctypes.c_int, [_P, ctypes.c_int32]),
    "sph_create_batch": (ctypes.c_int, [ctypes.POINTER(SphParams), _P, ctypes.c_int32, ctypes.POINTER(_P)]),
    "sph_num_scenes": (ctypes.c_int32, [_P]),
    "sph_get_scene_ranges": (ctypes.c_int, [_P, _P, _P]),
    "sph_get_scene_stats": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "sph_set_mlp": (ctypes.c_int, [_P, _P, ctypes.c_int32]),
    "sph_set_record_features": (ctypes.c_int, [_P, ctypes.c_int32]),
    "sph_get_features": (ctypes.c_int, [_P, _P, _P]),
    "sph_get_solve_start": (ctypes.c_int, [_P, _P]),
    "sph_get_grid": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "sph_mlp_train": (ctypes.c_int, [ctypes.POINTER(SphMlpTrainConfig), _P, _P, ctypes.c_int64, _P, _P]),
    "sph_mlp_eval": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, ctypes.c_int32, _P, _P]),
    "sph_boundary_psi_noalloc": (ctypes.c_int, [ctypes.POINTER(SphParams), _P, ctypes.c_int64, _P, _P, _P]),
    "sph_sample_solid": (ctypes.c_int, [_P, ctypes.c_int64, _P, ctypes.c_int64, _P, ctypes.c_int32, _P,
                                        ctypes.c_int32, _P, ctypes.c_int32, _P, _P, _P, ctypes.c_int64, _P,
                                        ctypes.c_int32]),
    "sph_num_fluid": (ctypes.c_int64, [_P]),
    "sph_num_boundary": (ctypes.c_int64, [_P]),
    "sph_stream": (ctypes.c_void_p, [_P]),
    "sph_synchronize": (ctypes.c_int, [_P]),
}

_LIB = None


def load(path: Path | str | None = None):
    """Load libwpsph.so and bind every entry point.  Raises if the library is absent."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -m warpsph_b200.build` (CUDA toolkit required); "
            "there is no CPU fallback")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def ptr(a: np.ndarray | None):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def check(ctx, rc: int):
    if rc != SPH_OK:
        msg = load().sph_last_error(ctx) if ctx else b""
        raise SphError(rc, (msg or b"").decode(errors="replace"))
