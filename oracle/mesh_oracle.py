"""CPU restatement of the solid mesh sampler (test infrastructure only).

Restates, in numpy float64 with the same operation order (numpy never fuses
multiply-adds), what ``sph_sample_solid`` computes on the GPU for the
reference's model sampler (wp_sph/solver/model.py:14-60): the lattice
``np.arange(lo, hi, spacing)`` per axis over the mesh bounds in meshgrid "ij"
order (model.py:21-24), an inside test per lattice point (the reference calls
trimesh's ``mesh.contains``; here: parity of the crossings of the +x ray with
the closed mesh, canonical edge functions, zeros resolved by perturbing the
query point by (e, e^2)), then ``points @ rot + pos`` (model.py:58-60) as
((p0 r0k + p1 r1k) + p2 r2k) + pos_k, cast to float32.
"""

from __future__ import annotations

import numpy as np


def _edge(py, pz, qy, qz, y, z):
    """Canonical edge function value and perturbed sign, elementwise."""
    swap = (py > qy) | ((py == qy) & (pz > qz))
    ay = np.where(swap, qy, py)
    az = np.where(swap, qz, pz)
    by = np.where(swap, py, qy)
    bz = np.where(swap, pz, qz)
    d1 = by - ay
    d2 = z - az
    d3 = bz - az
    d4 = y - ay
    v = d1 * d2 - d3 * d4
    s = np.sign(v)
    s = np.where(s == 0, np.where(d3 != 0, np.sign(-d3), np.sign(d1)), s)
    v = np.where(swap, -v, v)
    s = np.where(swap, -s, s)
    return v, s


def crossings(tri, y, z):
    """For triangles ``tri`` (k x 9: ax ay az bx by bz cx cy cz) and lines
    (y, z) (k each): (crosses, x of the crossing)."""
    ax, ay, az, bx, by, bz, cx, cy, cz = (tri[:, i] for i in range(9))
    e0, s0 = _edge(by, bz, cy, cz, y, z)
    e1, s1 = _edge(cy, cz, ay, az, y, z)
    e2, s2 = _edge(ay, az, by, bz, y, z)
    den = (e0 + e1) + e2
    ok = (s0 != 0) & (s0 == s1) & (s1 == s2) & (den != 0)
    with np.errstate(invalid="ignore", divide="ignore"):
        x = ax + (e1 * (bx - ax) + e2 * (cx - ax)) / den
    return ok, x


def sample_solid(verts, tris, spacing, rot=np.eye(3), pos=np.zeros(3)):
    verts = np.asarray(verts, np.float64)
    tris = np.asarray(tris, np.int64)
    lo, hi = verts.min(0), verts.max(0)
    xs, ys, zs = (np.arange(lo[a], hi[a], spacing) for a in range(3))
    T = np.concatenate([verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]], axis=1)
    nx, ny, nz = len(xs), len(ys), len(zs)
    inside = np.zeros((nx, ny, nz), bool)
    for iy in range(ny):
        yv = np.full(len(T), ys[iy])
        for iz in range(nz):
            ok, xh = crossings(T, yv, np.full(len(T), zs[iz]))
            h = np.sort(xh[ok])
            beyond = len(h) - np.searchsorted(h, xs, side="right")  # crossings with x_hit > x
            inside[:, iy, iz] = (beyond & 1).astype(bool)
    grid = np.stack(np.meshgrid(xs, ys, zs, indexing="ij"), -1).reshape(-1, 3)
    p = grid[inside.reshape(-1)]
    rot = np.asarray(rot, np.float64).reshape(3, 3)
    pos = np.asarray(pos, np.float64).reshape(3)
    out = np.empty((len(p), 3), np.float32)
    for k in range(3):
        out[:, k] = (((p[:, 0] * rot[0, k] + p[:, 1] * rot[1, k]) + p[:, 2] * rot[2, k]) + pos[k]).astype(np.float32)
    return out
