"""Headless frame output: positions recorded at FPS and written as PLY.

The reference renders a frame whenever ``sim_time - last_frame_time >=
frame_dt`` (IISPH.render, IISPH.py:1396-1406) into a USD stage (fluid points,
then the rigid boundary points, IISPH.py:1373-1394), and ``usd2ply.py``
converts each frame's first point set (the fluid) into a binary PLY with
``x, y, z`` (float32) and ``obj_id`` (uchar, 0) per vertex, named
``frame_<index>.ply`` and packed into one archive (usd2ply.py:12-92).  USD
and OpenGL are graphics stacks this package does without, so
``FrameRecorder`` keeps the frames in memory (written to ``.npz``) and
``export_ply`` writes the PLY files directly; the archive is a plain ``.tar``
(the reference compresses it with zstandard, which is not a dependency here).
"""

from __future__ import annotations

import tarfile
from pathlib import Path

import numpy as np

PLY_VERTEX = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("obj_id", "u1")])


class FrameRecorder:
    """Stand-in for the reference's UsdRenderer (IISPH.py:824-827): per
    rendered frame the simulated time, the fluid positions and the rigid
    boundary positions (boundary_x[boundary_hide_n:])."""

    def __init__(self, stage_path: str, fps: int):
        self.stage_path = stage_path
        self.fps = fps
        self.times: list[float] = []
        self.frames: list[np.ndarray] = []
        self.rigid: list[np.ndarray] = []

    def add(self, t: float, x: np.ndarray, rigid: np.ndarray | None = None):
        self.times.append(float(t))
        self.frames.append(np.asarray(x, np.float32))
        self.rigid.append(np.zeros((0, 3), np.float32) if rigid is None else np.asarray(rigid, np.float32))

    def save(self) -> str:
        path = self.stage_path if self.stage_path.endswith(".npz") else self.stage_path + ".npz"
        x = np.stack(self.frames) if self.frames else np.zeros((0, 0, 3), np.float32)
        rigid = np.stack(self.rigid) if self.rigid else np.zeros((0, 0, 3), np.float32)
        np.savez_compressed(path, times=np.asarray(self.times), x=x, rigid=rigid)
        return path


def write_ply(path, points, obj_id: int = 0):
    """Binary little-endian PLY of ``points`` (n x 3) with a constant obj_id,
    the vertex layout of usd2ply.py:26-31."""
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    v = np.empty(len(pts), PLY_VERTEX)
    v["x"], v["y"], v["z"] = pts[:, 0], pts[:, 1], pts[:, 2]
    v["obj_id"] = obj_id
    header = ("ply\nformat binary_little_endian 1.0\n"
              f"element vertex {len(pts)}\n"
              "property float x\nproperty float y\nproperty float z\nproperty uchar obj_id\nend_header\n")
    with open(path, "wb") as f:
        f.write(header.encode("ascii"))
        f.write(v.tobytes())


def read_ply(path) -> np.ndarray:
    """The vertices of a PLY written by write_ply (structured PLY_VERTEX)."""
    data = Path(path).read_bytes()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    head = data[:end].decode("ascii").splitlines()
    if head[1] != "format binary_little_endian 1.0":
        raise ValueError(f"{path}: not a binary little-endian PLY")
    n = int(next(h for h in head if h.startswith("element vertex")).split()[2])
    return np.frombuffer(data, PLY_VERTEX, count=n, offset=end)


def export_ply(frames, out_dir, archive: str | None = None) -> list[Path]:
    """One PLY per recorded frame (frame_0000.ply, ...; usd2ply.py:36-43)
    from a FrameRecorder, an ``.npz`` it saved, or a list of position arrays;
    with ``archive``, the files are also packed into that ``.tar``."""
    if isinstance(frames, FrameRecorder):
        xs = frames.frames
    elif isinstance(frames, (str, Path)):
        xs = list(np.load(frames)["x"])
    else:
        xs = list(frames)
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    paths = []
    for k, x in enumerate(xs):
        p = out / f"frame_{k:04d}.ply"
        write_ply(p, x, obj_id=0)
        paths.append(p)
    if archive:
        with tarfile.open(archive, "w") as tar:
            for p in paths:
                tar.add(p, arcname=p.name)
    return paths
