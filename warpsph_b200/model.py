"""Mesh models as boundary particles (wp_sph/solver/model.py:14-60).

``load_model(filename, scale, pos, rot, spacing)`` keeps the reference's
signature and result: the lattice ``np.arange(lo, hi, spacing)`` per axis over
the scaled mesh's bounds, in meshgrid "ij" order, restricted to the points
inside the closed mesh, then ``points @ rot + pos``.  The inside test and the
transform run on the GPU (``sph_sample_solid`` in libwpsph.so: ray-crossing
parity along +x, one block per lattice line); the reference's trimesh /
joblib stack is replaced by a small OBJ reader and an ``.npz`` cache of the
sampled points.  The procedural meshes (box, torus, UV sphere) are closed
triangle meshes for scenes and tests.
"""

from __future__ import annotations

import ctypes
import hashlib
import os
from pathlib import Path

import numpy as np

from . import _lib

CACHE_DIR = Path(os.environ.get("WPSPH_MODEL_CACHE", Path(__file__).resolve().parent / ".model_cache"))


# ------------------------------------------------------------------ meshes

def load_obj(path) -> tuple[np.ndarray, np.ndarray]:
    """Vertices (float64, n x 3) and triangles (int32, m x 3) of an OBJ file.
    Polygons are split into triangle fans; ``v/vt/vn`` references and
    negative (relative) indices are accepted; other records are ignored."""
    verts, faces = [], []
    with open(path, "r", errors="replace") as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "v" and len(parts) >= 4:
                verts.append([float(parts[1]), float(parts[2]), float(parts[3])])
            elif parts[0] == "f" and len(parts) >= 4:
                idx = []
                for tok in parts[1:]:
                    k = int(tok.split("/")[0])
                    idx.append(k - 1 if k > 0 else len(verts) + k)
                for t in range(1, len(idx) - 1):
                    faces.append([idx[0], idx[t], idx[t + 1]])
    v = np.asarray(verts, np.float64).reshape(-1, 3)
    t = np.asarray(faces, np.int32).reshape(-1, 3)
    if t.size and (t.min() < 0 or t.max() >= len(v)):
        raise ValueError(f"{path}: face index out of range")
    return v, t


def save_obj(path, verts, tris):
    with open(path, "w") as f:
        for p in np.asarray(verts, np.float64):
            f.write(f"v {float(p[0])!r} {float(p[1])!r} {float(p[2])!r}\n")
        for t in np.asarray(tris, np.int64):
            f.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


def box_mesh(lo, hi):
    """Closed axis-aligned box, 12 triangles, outward normals."""
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    v = np.array([[lo[0] if i & 1 == 0 else hi[0], lo[1] if i & 2 == 0 else hi[1], lo[2] if i & 4 == 0 else hi[2]]
                  for i in range(8)])
    t = np.array([[0, 2, 1], [1, 2, 3], [4, 5, 6], [5, 7, 6], [0, 1, 4], [1, 5, 4],
                  [2, 6, 3], [3, 6, 7], [0, 4, 2], [2, 4, 6], [1, 3, 5], [3, 7, 5]], np.int32)
    return v, t


def torus_mesh(center, major, minor, n_major=32, n_minor=16, axis="y"):
    """Closed triangulated torus around ``axis`` through ``center``."""
    u = 2 * np.pi * np.arange(n_major) / n_major
    w = 2 * np.pi * np.arange(n_minor) / n_minor
    uu, ww = np.meshgrid(u, w, indexing="ij")
    rr = major + minor * np.cos(ww)
    a = rr * np.cos(uu)
    b = rr * np.sin(uu)
    c = minor * np.sin(ww)
    pts = {"y": np.stack([a, c, b], -1), "z": np.stack([a, b, c], -1), "x": np.stack([c, a, b], -1)}[axis]
    v = pts.reshape(-1, 3) + np.asarray(center, np.float64)
    i, j = np.meshgrid(np.arange(n_major), np.arange(n_minor), indexing="ij")
    p00 = i * n_minor + j
    p10 = ((i + 1) % n_major) * n_minor + j
    p01 = i * n_minor + (j + 1) % n_minor
    p11 = ((i + 1) % n_major) * n_minor + (j + 1) % n_minor
    t = np.concatenate([np.stack([p00, p10, p11], -1).reshape(-1, 3), np.stack([p00, p11, p01], -1).reshape(-1, 3)])
    return v, t.astype(np.int32)


def sphere_mesh(center, radius, n_lat=16, n_lon=32):
    """Closed UV sphere (poles as single vertices)."""
    th = np.pi * np.arange(1, n_lat) / n_lat
    ph = 2 * np.pi * np.arange(n_lon) / n_lon
    tt, pp = np.meshgrid(th, ph, indexing="ij")
    ring = np.stack([np.sin(tt) * np.cos(pp), np.cos(tt), np.sin(tt) * np.sin(pp)], -1).reshape(-1, 3)
    v = np.concatenate([[[0, 1, 0]], ring, [[0, -1, 0]]]) * radius + np.asarray(center, np.float64)
    top, bot = 0, len(v) - 1
    tris = []
    for k in range(n_lon):
        k2 = (k + 1) % n_lon
        tris.append([top, 1 + k2, 1 + k])
        for r in range(n_lat - 2):
            a, b = 1 + r * n_lon + k, 1 + r * n_lon + k2
            c, d = a + n_lon, b + n_lon
            tris += [[a, b, d], [a, d, c]]
        base = 1 + (n_lat - 2) * n_lon
        tris.append([base + k, base + k2, bot])
    return v, np.asarray(tris, np.int32)


# ------------------------------------------------------------------ sampling

def lattice(verts, spacing):
    """The reference's lattice axes over the mesh bounds (model.py:21-24)."""
    lo, hi = verts.min(0), verts.max(0)
    return [np.arange(lo[a], hi[a], spacing) for a in range(3)]


def sample_solid(verts, tris, spacing, rot=np.eye(3), pos=np.zeros(3), device=0) -> np.ndarray:
    """Lattice points inside the closed mesh, ``points @ rot + pos``, float32,
    in the reference's lattice order (x slowest, z fastest)."""
    verts = np.ascontiguousarray(verts, np.float64)
    tris = np.ascontiguousarray(tris, np.int32)
    xs, ys, zs = (np.ascontiguousarray(a, np.float64) for a in lattice(verts, spacing))
    rot = np.ascontiguousarray(np.asarray(rot, np.float64).reshape(3, 3))
    pos = np.ascontiguousarray(np.asarray(pos, np.float64).reshape(3))
    cap = max(len(xs) * len(ys) * len(zs), 1)
    out = np.zeros((cap, 3), np.float32)
    count = ctypes.c_int64(0)
    L = _lib.load()
    rc = L.sph_sample_solid(_lib.ptr(verts), len(verts), _lib.ptr(tris), len(tris), _lib.ptr(xs), len(xs),
                            _lib.ptr(ys), len(ys), _lib.ptr(zs), len(zs), _lib.ptr(rot), _lib.ptr(pos),
                            _lib.ptr(out), cap, ctypes.byref(count), int(device))
    _lib.check(None, rc)
    return out[: count.value].copy()


def model_dir(filename):
    try:
        from wp_sph.main import model_dir as md

        return md(filename)
    except ImportError:
        return Path(filename)


def load_model(filename, scale=1.0, pos=np.zeros(3), rot=np.eye(3), spacing=None, device=0):
    """model.py:53-60: the mesh file's solid, sampled at ``spacing``
    (default DIAMETER), rotated and moved.  Results are cached on disk by the
    file's contents and the arguments."""
    if spacing is None:
        try:
            from wp_sph.main import DIAMETER as spacing
        except ImportError:
            spacing = 0.05
    path = Path(filename)
    if not path.exists():
        path = Path(model_dir(filename))
    data = path.read_bytes()
    key = hashlib.sha256(data + np.asarray([scale, spacing], np.float64).tobytes()
                         + np.asarray(rot, np.float64).tobytes() + np.asarray(pos, np.float64).tobytes()).hexdigest()
    cached = CACHE_DIR / f"{path.stem}_{key[:16]}.npz"
    if cached.exists():
        return np.load(cached)["points"]
    verts, tris = load_obj(path)
    pts = sample_solid(verts * float(scale), tris, float(spacing), rot, pos, device=device)
    CACHE_DIR.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(cached, points=pts)
    return pts
