"""B200-native (sm_100a) IISPH time step behind the wp_sph solver API.

The compute path is libwpsph.so (CUDA, C ABI in include/wpsph.h), loaded
through ctypes by ``warpsph_b200.solver.IISPH``; importing this package does
not touch the GPU.
"""
from .params import PRESETS, SolverParams, preset_params  # noqa: F401

__all__ = ["SolverParams", "PRESETS", "preset_params", "IISPH"]


def __getattr__(name):
    if name == "IISPH":
        from .solver import IISPH

        return IISPH
    raise AttributeError(name)
