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
    """Particles on the six faces of the box [lo, hi]: the points of a lattice
    with round((hi - lo) / spacing) + 1 (at least 2) evenly spaced planes per
    axis, from lo to hi, that lie on a face; ordered x, y, z (z fastest)."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    n = [max(2, int(round((h - l) / spacing)) + 1) for l, h in zip(lo, hi)]
    grids = [np.linspace(l, h, k) for l, h, k in zip(lo, hi, n)]
    ix, iy, iz = (a.ravel() for a in np.meshgrid(*[np.arange(k) for k in n], indexing="ij"))
    face = (ix == 0) | (ix == n[0] - 1) | (iy == 0) | (iy == n[1] - 1) | (iz == 0) | (iz == n[2] - 1)
    pts = np.stack([grids[0][ix[face]], grids[1][iy[face]], grids[2][iz[face]]], axis=1)
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


def _inside_box(pts, lo, hi, margin):
    return np.all((pts > np.asarray(lo) + margin) & (pts < np.asarray(hi) - margin), axis=1)


def _inside_torus(pts, center, major, minor, axis, margin):
    d = pts.astype(np.float64) - np.asarray(center, np.float64)
    along = d[:, axis]
    plane = np.delete(d, axis, axis=1)
    ring = np.sqrt(np.sum(plane * plane, axis=1)) - major
    return ring * ring + along * along < (minor - margin) ** 2


def pour_obstacles(seed=2, spacing=0.008, boxes=6, tori=4, lo=(0.45, 0.25, 0.45), hi=(1.55, 1.2, 1.55),
                   rmin=0.05, rmax=0.2):
    """A seeded procedural obstacle: the union of `boxes` axis-aligned boxes
    (half-extents uniform in [rmin, rmax] per axis) and `tori` tori (major
    radius uniform in [rmin, rmax], tube radius 0.3-0.5 of it, axis x, y or z),
    centres uniform in [lo, hi], surface-sampled at `spacing` (box_surface,
    torus_surface).  Surface particles inside another shape are dropped, so
    the particles sample the union's surface."""
    rng = np.random.default_rng(seed)
    shapes = []
    for _ in range(boxes):
        c = rng.uniform(lo, hi)
        half = rng.uniform(rmin, rmax, size=3)
        shapes.append(("box", c - half, c + half))
    for _ in range(tori):
        c = rng.uniform(lo, hi)
        major = float(rng.uniform(rmin, rmax))
        minor = max(2.0 * spacing, major * float(rng.uniform(0.3, 0.5)))
        shapes.append(("torus", c, major, minor, int(rng.integers(0, 3))))
    parts = []
    for k, sh in enumerate(shapes):
        pts = box_surface(sh[1], sh[2], spacing) if sh[0] == "box" else torus_surface(sh[1], sh[2], sh[3], spacing,
                                                                                          axis=sh[4])
        keep = np.ones(len(pts), bool)
        for m, other in enumerate(shapes):
            if m == k:
                continue
            if other[0] == "box":
                keep &= ~_inside_box(pts, other[1], other[2], 0.5 * spacing)
            else:
                keep &= ~_inside_torus(pts, other[1], other[2], other[3], other[4], 0.5 * spacing)
        parts.append(pts[keep])
    return np.concatenate(parts).astype(np.float32), shapes


class Inlet:
    """A rectangular opening emitting fluid at a fixed speed along -y: a layer
    of particles on a `spacing` lattice over the opening each time the previous
    layer has moved one spacing on, i.e. every spacing / speed seconds, until
    `max_particles` have been emitted.  Layer k leaves the opening at
    t_k = k spacing / speed; at time t it is emitted (t - t_k) speed below the
    opening with velocity speed along -y.  Seeded uniform jitter in
    [-jitter, jitter] per coordinate."""

    def __init__(self, center=(1.0, 1.8, 1.0), size=(0.3, 0.3), spacing=0.008, speed=2.0,
                 max_particles=2_000_000, jitter=5e-5, seed=2):
        nx, nz = int(round(size[0] / spacing)), int(round(size[1] / spacing))
        ix, iz = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij"))
        self.offsets = np.stack([(ix - (nx - 1) / 2.0) * spacing, np.zeros(len(ix)), (iz - (nz - 1) / 2.0) * spacing],
                                axis=1)
        self.center = np.asarray(center, np.float64)
        self.spacing, self.speed = float(spacing), float(speed)
        self.period = self.spacing / self.speed
        self.max_particles = int(max_particles)
        self.jitter = float(jitter)
        self.rng = np.random.default_rng(seed)
        self.layers = 0
        self.emitted = 0

    @property
    def layer_size(self) -> int:
        return len(self.offsets)

    @property
    def done(self) -> bool:
        return self.emitted >= self.max_particles

    def due(self, t: float):
        """Particles of every layer whose emission time is <= t and that has not
        been emitted yet: (x, v), float32 arrays of shape (m, 3)."""
        xs = []
        while not self.done and self.layers * self.period <= t + 1e-12:
            lag = t - self.layers * self.period
            pts = self.center + self.offsets - np.array([0.0, lag * self.speed, 0.0])
            if self.jitter > 0:
                pts = pts + self.rng.uniform(-self.jitter, self.jitter, size=pts.shape)
            pts = pts[: self.max_particles - self.emitted]
            xs.append(pts)
            self.layers += 1
            self.emitted += len(pts)
        if not xs:
            return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32)
        x = np.concatenate(xs).astype(np.float32)
        v = np.zeros_like(x)
        v[:, 1] = -self.speed
        return x, v


def pour_scene(seed=2, spacing=0.008, domain=(2.0, 2.0, 2.0), layers=2):
    """Fluid poured onto a procedural obstacle: a 2 x 2 x 2 m box walled by
    `layers` boundary layers at `spacing`, the seeded obstacle union of
    `pour_obstacles`, and the inlet's first layer as the initial fluid.
    Returns (scene, inlet); feed inlet.due(sim_time) to IISPH.add_fluid."""
    walls = box_boundary(domain, spacing, layers)
    obstacle, _ = pour_obstacles(seed=seed, spacing=spacing)
    inlet = Inlet(center=(domain[0] / 2, domain[1] * 0.9, domain[2] / 2), spacing=spacing, seed=seed)
    x, v = inlet.due(0.0)
    scene = Scene(fluid_x=x, fluid_v=v, boundary_x=walls.astype(np.float32), boundary_hide_n=len(walls),
                  box=tuple(domain))
    return add_obstacles(scene, [obstacle]), inlet


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
