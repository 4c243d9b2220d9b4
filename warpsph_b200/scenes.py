"""Particle scene construction (host side).

``box_scene`` restates the reference's ``IISPH.init_particles``
(IISPH.py:857-1000) with numpy instead of Python loops, producing the same
particles in the same order.  ``dam_break`` builds the benchmark scenes: a fluid
block on the cubic lattice at indices [0, n) per axis with seeded uniform
jitter, in a box walled by boundary lattice layers (same lattice convention).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Scene:
    fluid_x: np.ndarray          # (n, 3) float32
    fluid_v: np.ndarray          # (n, 3) float32
    boundary_x: np.ndarray       # (nb, 3) float32
    boundary_hide_n: int         # boundary particles that belong to the box walls
    box: tuple

    @property
    def n(self) -> int:
        return len(self.fluid_x)

    @property
    def boundary_n(self) -> int:
        return len(self.boundary_x)


def box_boundary(box, spacing, layers) -> np.ndarray:
    """Wall lattice of IISPH.py:872-912: indices [-L, N+L) per axis minus the
    interior [0, N), N = int(BOX / spacing), loop order x, y, z (z fastest)."""
    dims = [int(b / spacing) for b in box]
    axes = [np.arange(-layers, d + layers) for d in dims]
    ix, iy, iz = np.meshgrid(*axes, indexing="ij")
    ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
    outside = ((ix < 0) | (ix > dims[0] - 1) | (iy < 0) | (iy > dims[1] - 1) | (iz < 0) | (iz > dims[2] - 1))
    pts = np.stack([ix[outside] * spacing, iy[outside] * spacing, iz[outside] * spacing], axis=1)
    return pts


def box_scene(box, spacing, min_point=None, max_point=None, fluid_depth=0.0, boundary_layers=3) -> Scene:
    """IISPH.init_particles (IISPH.py:857-1000) for the EMPTY scene type."""
    assert spacing > 0, "Particle spacing must be positive"
    dims = [int(b / spacing) for b in box]
    boundary = box_boundary(box, spacing, boundary_layers)
    fluid = []
    if fluid_depth > 0:
        # pool particles (IISPH.py:915-925): interior lattice up to fluid_depth,
        # minus the rectangle's neighbourhood
        fluid_y_max = int(fluid_depth / spacing)
        axes = [np.arange(0, d) for d in dims]
        ix, iy, iz = (a.ravel() for a in np.meshgrid(*axes, indexing="ij"))
        keep = iy <= fluid_y_max
        pts = np.stack([ix * spacing, iy * spacing, iz * spacing], axis=1)[keep]
        if min_point is not None and max_point is not None:
            lo = np.asarray(min_point) - spacing
            hi = np.asarray(max_point) + spacing
            in_rect = np.all((pts > lo) & (pts < hi), axis=1)
            pts = pts[~in_rect]
        fluid.append(pts)
    if min_point is not None and max_point is not None:
        for a in range(3):
            assert 0 < min_point[a] < max_point[a] < box[a], "Invalid range for rectangle"
        xr = np.arange(min_point[0], max_point[0], spacing)
        yr = np.arange(min_point[1], max_point[1], spacing)
        zr = np.arange(min_point[2], max_point[2], spacing)
        xx, yy, zz = np.meshgrid(xr, yr, zr, indexing="ij")
        fluid.append(np.stack([xx.ravel(), yy.ravel(), zz.ravel()]).T)
    fx = np.concatenate(fluid).astype(np.float32) if fluid else np.zeros((0, 3), np.float32)
    return Scene(fluid_x=fx, fluid_v=np.zeros_like(fx), boundary_x=boundary.astype(np.float32),
                 boundary_hide_n=len(boundary), box=tuple(box))


def reference_empty_scene(box=(4.0, 4.0, 4.0), spacing=0.05) -> Scene:
    """The reference's default scene (SceneType.EMPTY, IISPH.py:763-766)."""
    bw, bh, bl = box
    min_point = (bw * 0.02, bh * 0.02, bl * 0.02)
    max_point = (bw * 0.98, bh * 0.4, bl * 0.55)
    return box_scene(box, spacing, min_point, max_point)


def dam_break(fluid=(20, 20, 20), spacing=0.02, box=(1.0, 0.6, 0.4), jitter=1e-4, layers=2,
              seed=0, velocity=(0.0, 0.0, 0.0)) -> Scene:
    """Fluid block at lattice indices [0, n) per axis (positions i * spacing)
    plus i.i.d. uniform jitter in [-jitter, jitter] per coordinate from
    numpy.random.default_rng(seed); walls as in ``box_boundary``."""
    rng = np.random.default_rng(seed)
    axes = [np.arange(n) for n in fluid]
    ix, iy, iz = (a.ravel() for a in np.meshgrid(*axes, indexing="ij"))
    x = np.stack([ix * spacing, iy * spacing, iz * spacing], axis=1)
    if jitter > 0:
        x = x + rng.uniform(-jitter, jitter, size=x.shape)
    v = np.zeros_like(x) + np.asarray(velocity, dtype=np.float64)
    b = box_boundary(box, spacing, layers)
    return Scene(fluid_x=x.astype(np.float32), fluid_v=v.astype(np.float32),
                 boundary_x=b.astype(np.float32), boundary_hide_n=len(b), box=tuple(box))


def box_surface(lo, hi, spacing) -> np.ndarray:
    """Particles on the six faces of the box [lo, hi]: every lattice point
    lo + k * spacing (k >= 0, up to hi) with at least one coordinate on a face,
    ordered x, y, z (z fastest)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    n = [int(np.floor((h - l) / spacing + 1e-9)) + 1 for l, h in zip(lo, hi)]
    ix, iy, iz = (a.ravel() for a in np.meshgrid(*[np.arange(k) for k in n], indexing="ij"))
    face = (ix == 0) | (ix == n[0] - 1) | (iy == 0) | (iy == n[1] - 1) | (iz == 0) | (iz == n[2] - 1)
    pts = lo + spacing * np.stack([ix[face], iy[face], iz[face]], axis=1)
    return pts.astype(np.float32)


def torus_surface(center, major, minor, spacing, axis=1) -> np.ndarray:
    """Particles on a torus surface: a tube of radius ``minor`` around a circle
    of radius ``major`` in the plane normal to ``axis`` (0, 1, 2 = x, y, z),
    about ``spacing`` apart along the circle (at its centre line) and around
    the tube."""
    nu = max(8, int(round(2 * np.pi * major / spacing)))
    nv = max(6, int(round(2 * np.pi * minor / spacing)))
    u = 2 * np.pi * np.arange(nu) / nu
    w = 2 * np.pi * np.arange(nv) / nv
    uu, ww = (a.ravel() for a in np.meshgrid(u, w, indexing="ij"))
    ring = major + minor * np.cos(ww)
    a, b, c = ring * np.cos(uu), minor * np.sin(ww), ring * np.sin(uu)  # b runs along the axis
    local = {0: (b, a, c), 1: (a, b, c), 2: (a, c, b)}[axis]
    pts = np.stack(local, axis=1) + np.asarray(center, np.float64)
    return pts.astype(np.float32)


def add_obstacles(scene: Scene, obstacles) -> Scene:
    """Append obstacle boundary particles after the box walls (the walls stay
    the first boundary_hide_n boundary particles, as in IISPH.py:927)."""
    extra = [np.asarray(o, np.float32).reshape(-1, 3) for o in obstacles]
    bx = np.concatenate([scene.boundary_x] + extra).astype(np.float32)
    return Scene(scene.fluid_x, scene.fluid_v, bx, scene.boundary_hide_n, scene.box)


def preset_scene(name: str) -> Scene:
    from .params import PRESETS

    c = PRESETS[name]
    return dam_break(fluid=c["fluid"], spacing=c["diameter"], box=c["box"], jitter=c["jitter"],
                     layers=c["layers"], seed=c["seed"])


def batched_scenes(count=64, seed=3, spacing=0.01, jitter=5e-5, layers=2):
    """Independent dam breaks for batched solving: fluid counts log-uniform in
    [5k, 200k], box aspect ratios uniform in [1, 3] per axis, fluid fill
    fraction uniform in [0.2, 0.5] (seeded).  The fluid block sits in the box
    corner with the box's proportions scaled by fill^(1/3)."""
    rng = np.random.default_rng(seed)
    scenes = []
    for k in range(count):
        n_target = float(np.exp(rng.uniform(np.log(5e3), np.log(2e5))))
        aspect = rng.uniform(1.0, 3.0, size=3)
        fill = float(rng.uniform(0.2, 0.5))
        v_box = n_target * spacing**3 / fill
        box = aspect * (v_box / float(np.prod(aspect))) ** (1.0 / 3.0)
        nf = [max(2, int(round(fill ** (1.0 / 3.0) * b / spacing))) for b in box]
        box = tuple(float(max(b, (n + 1) * spacing)) for b, n in zip(box, nf))
        scenes.append(dam_break(fluid=tuple(nf), spacing=spacing, box=box, jitter=jitter, layers=layers,
                                seed=seed * 1000 + k))
    return scenes
