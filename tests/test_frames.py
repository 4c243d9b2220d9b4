"""Headless frame output on the CPU: the PLY layout of usd2ply.py:26-31 and
the render cadence of IISPH.render (IISPH.py:1396-1406)."""
import tarfile
from types import SimpleNamespace

import numpy as np

from warpsph_b200.frames import FrameRecorder, PLY_VERTEX, export_ply, read_ply, write_ply


def test_ply_layout_round_trip(tmp_path):
    pts = np.random.default_rng(0).normal(size=(257, 3)).astype(np.float32)
    p = tmp_path / "a.ply"
    write_ply(p, pts)
    raw = p.read_bytes()
    head = raw[: raw.index(b"end_header\n") + len(b"end_header\n")].decode()
    assert head == ("ply\nformat binary_little_endian 1.0\nelement vertex 257\nproperty float x\n"
                    "property float y\nproperty float z\nproperty uchar obj_id\nend_header\n")
    assert len(raw) == len(head) + 257 * 13 and PLY_VERTEX.itemsize == 13
    v = read_ply(p)
    assert np.array_equal(np.stack([v["x"], v["y"], v["z"]], 1), pts)
    assert np.all(v["obj_id"] == 0)


def test_export_frames_and_archive(tmp_path):
    rec = FrameRecorder(str(tmp_path / "run"), 60)
    frames = [np.full((5 + k, 3), k, np.float32) for k in range(3)]
    for k, f in enumerate(frames):
        rec.add(k / 60, f)
    paths = export_ply(rec, tmp_path / "ply", archive=str(tmp_path / "run.tar"))
    assert [p.name for p in paths] == ["frame_0000.ply", "frame_0001.ply", "frame_0002.ply"]
    for p, f in zip(paths, frames):
        v = read_ply(p)
        assert len(v) == len(f) and np.all(v["x"] == f[:, 0])
    with tarfile.open(tmp_path / "run.tar") as tar:
        assert sorted(tar.getnames()) == [p.name for p in paths]


def _fake_solver(times, recorder, fps=60):
    """The attributes IISPH.render reads, with positions that name the step."""
    s = SimpleNamespace(frame_dt=1.0 / fps, sim_time=0.0, last_frame_time=0.0, renderer=recorder,
                        boundary_hide_n=2, previewer=None)
    s.x = SimpleNamespace(numpy=lambda: np.full((3, 3), s.sim_time, np.float32))
    s.boundary_x = SimpleNamespace(numpy=lambda: np.zeros((4, 3), np.float32))
    return s


def test_render_cadence_rule(tmp_path):
    """A frame whenever sim_time - last_frame_time >= 1/FPS, checked against
    the rule applied to the same time sequence (dt = 5e-4 s: every 34th step)."""
    from warpsph_b200.solver import IISPH

    rec = FrameRecorder(str(tmp_path / "run"), 60)
    s = _fake_solver(None, rec)
    dt = 5e-4
    want, last = [], 0.0
    for k in range(1, 501):
        s.sim_time = k * dt
        IISPH.render(s)
        if k * dt - last >= 1.0 / 60:
            want.append(k * dt)
            last = k * dt
    assert rec.times == want and len(want) == 14
    assert all(np.all(f == np.float32(t)) for f, t in zip(rec.frames, rec.times))
    assert all(r.shape == (2, 3) for r in rec.rigid)
    path = rec.save()
    d = np.load(path)
    assert np.array_equal(d["times"], np.asarray(want)) and d["x"].shape == (14, 3, 3)
