"""Solver parameters: the runtime form of the reference's module constants.

The reference bakes its constants into Warp kernels at import
(wp_sph/main.py:25-61, sph_funcs.py:43-44); here they are fields of
``SolverParams`` with the same defaults, converted to the C struct ``SphParams``
of include/wpsph.h.  Derived values use the reference's formulas
(main.py:57-61) evaluated in Python float64, so they are bit-identical.
"""

from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

from . import _lib

WARM_MODES = {"zero": _lib.SPH_WARM_ZERO, "half": _lib.SPH_WARM_HALF, "mlp": _lib.SPH_WARM_MLP}


@dataclass
class SolverParams:
    diameter: float = 0.05        # DIAMETER (main.py:26)
    rho0: float = 1.0e3           # RHO_0 (main.py:30)
    gravity: float = 9.8          # GRAVITY (main.py:25)
    omega: float = 0.5            # OMEGA (main.py:27)
    eta: float = 1.0e-3           # ETA (main.py:28)
    inv_small: float = 1.0e-6     # INV_SMALL (main.py:29)
    vis_mu_scale: float = 0.0     # VIS_MU = vis_mu_scale * RHO_0 (main.py:61)
    w_table_size: int = 8192      # W_SIZE (sph_funcs.py:43)
    g_table_size: int = 65536     # GRAD_W_SIZE (sph_funcs.py:44)
    min_iter: int = 2             # IISPH.py:1201
    max_loop: int = 100           # IISPH.py:1202
    fixed_iters: int = -1
    warm_start: str = "zero"      # "zero" (IISPH.py:173) | "half" (IISPH.py:174) | "mlp"
    max_ff: int = 48
    max_fb: int = 48
    keep_fb_lists: bool = False
    use_graph: bool = True
    device: int = 0
    block_size: int = 0           # neighbour build threads per block (0 = 128)
    timeout_ms: int = 2000
    jacobi_block: int = 0         # pressure solve threads per block (0 = 1024)
    jacobi_ppt: int = 0           # particles per solve thread (0 = 1)
    jacobi_unroll: int = 0        # solve neighbour-loop unroll (0 = 4)
    move_boundary: bool = False   # boundary moves with its velocities (DYNAMIC_SCENE, main.py:20)
    warm_continue: bool = False   # "mlp": a step after a capped solve starts from that solve's pressure
    plain_loads: bool = False     # neighbour gathers: plain loads instead of the texture path
    dt0: float | None = None      # None: TIME_STEP_MAX (IISPH.py:747)
    domain_min: tuple = (0.0, 0.0, 0.0)
    domain_max: tuple = (0.0, 0.0, 0.0)
    extra: dict = field(default_factory=dict)

    # derived (main.py:57-61)
    @property
    def h(self) -> float:
        return 2 * self.diameter

    @property
    def fluid_mass(self) -> float:
        return self.rho0 * self.diameter**3

    @property
    def sigma(self) -> float:
        return 8 / (math.pi * self.h**3)

    @property
    def dt_max(self) -> float:
        return 5e-2 * self.diameter

    @property
    def cfl_len(self) -> float:
        return 0.4 * self.diameter

    @property
    def vis_mu(self) -> float:
        return self.vis_mu_scale * self.rho0

    def replace(self, **kw) -> "SolverParams":
        return dataclasses.replace(self, **kw)

    def to_c(self) -> _lib.SphParams:
        p = _lib.SphParams()
        p.spacing = self.diameter
        p.h = self.h
        p.rho0 = self.rho0
        p.gravity = self.gravity
        p.omega = self.omega
        p.eta = self.eta
        p.inv_small = self.inv_small
        p.vis_mu = self.vis_mu
        p.fluid_mass = self.fluid_mass
        p.sigma = self.sigma
        p.dt_max = self.dt_max
        p.cfl_len = self.cfl_len
        p.dt0 = self.dt_max if self.dt0 is None else self.dt0
        for a in range(3):
            p.domain_min[a] = self.domain_min[a]
            p.domain_max[a] = self.domain_max[a]
        p.w_table_size = self.w_table_size
        p.g_table_size = self.g_table_size
        p.min_iter = self.min_iter
        p.max_loop = self.max_loop
        p.fixed_iters = self.fixed_iters
        p.warm_start = WARM_MODES[self.warm_start]
        p.max_ff = self.max_ff
        p.max_fb = self.max_fb
        p.keep_fb_lists = int(self.keep_fb_lists)
        p.use_graph = int(self.use_graph)
        p.device = self.device
        p.block_size = self.block_size
        p.timeout_ms = self.timeout_ms
        p.jacobi_block = self.jacobi_block
        p.jacobi_ppt = self.jacobi_ppt
        p.jacobi_unroll = self.jacobi_unroll
        p.move_boundary = int(self.move_boundary)
        p.warm_continue = int(self.warm_continue)
        p.plain_loads = int(self.plain_loads)
        return p

    @classmethod
    def from_reference_module(cls, main, **kw) -> "SolverParams":
        """Defaults read from a ``wp_sph.main``-style constants module."""
        return cls(diameter=main.DIAMETER, rho0=main.RHO_0, gravity=main.GRAVITY, omega=main.OMEGA,
                   eta=main.ETA, inv_small=main.INV_SMALL,
                   vis_mu_scale=getattr(main, "VIS_MU_SCALE", 0.0), **kw)


# Scene presets for the benchmark workloads: dam breaks on a cubic lattice
# with seeded jitter, 2 boundary layers, 1024-sample kernel tables, g = 9.81.
PRESETS = {
    "dam_break_8k": dict(diameter=0.02, fluid=(20, 20, 20), box=(1.0, 0.6, 0.4), jitter=1e-4,
                         layers=2, steps=200, seed=0),
    "dam_break_1m": dict(diameter=0.01, fluid=(100, 100, 100), box=(2.0, 1.0, 1.0), jitter=5e-5,
                         layers=2, steps=500, seed=1),
}


# Fluid poured from a 0.3 x 0.3 m inlet at 2 m/s onto a procedural obstacle
# in a 2 m cube (scenes.pour_scene): 0.008 m spacing, dt = 4e-4 s, until 2M fluid.
POUR = dict(diameter=0.008, domain=(2.0, 2.0, 2.0), layers=2, max_particles=2_000_000, seed=2, steps=1000)


def pour_params(**kw) -> SolverParams:
    d = POUR["diameter"] * (POUR["layers"] + 1)
    lo = tuple(-d for _ in range(3))
    hi = tuple(b + d for b in POUR["domain"])
    base = dict(diameter=POUR["diameter"], gravity=9.81, w_table_size=1024, g_table_size=1024,
                domain_min=lo, domain_max=hi)
    base.update(kw)
    return SolverParams(**base)


def preset_params(name: str, **kw) -> SolverParams:
    cfg = PRESETS[name]
    base = dict(diameter=cfg["diameter"], gravity=9.81, w_table_size=1024, g_table_size=1024)
    base.update(kw)
    return SolverParams(**base)
