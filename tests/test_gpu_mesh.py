"""Solid mesh sampling on the GPU (sph_sample_solid) against its CPU
restatement (oracle/mesh_oracle.py), bit for bit, on closed procedural meshes;
the reference's model sampler is wp_sph/solver/model.py:14-60."""
import numpy as np
import pytest

from oracle import mesh_oracle as MO

pytestmark = pytest.mark.gpu

HAND_ROT = np.array([[np.cos(np.radians(160)), -np.sin(np.radians(160)), 0],
                     [np.sin(np.radians(160)), np.cos(np.radians(160)), 0], [0, 0, 1]])
PLANE_ROT = np.array([[1, 0, 0], [0, 0, -1], [0, 1, 0]], np.float64)


def _meshes():
    from warpsph_b200.model import box_mesh, sphere_mesh, torus_mesh

    return {
        "box": (box_mesh((0.1, 0.2, 0.3), (0.5, 0.45, 0.7)), 0.02, np.eye(3), np.zeros(3)),
        "torus": (torus_mesh((0.0, 0.0, 0.0), 0.3, 0.1, 48, 24), 0.01, HAND_ROT, np.array([4.5, 2.0, 1.0])),
        "sphere": (sphere_mesh((0.1, 0.1, 0.1), 0.2), 0.01, PLANE_ROT, np.array([0.0, 4.0, 4.0])),
        # a lattice line through the sphere's poles and along its seams
        "sphere_on_lattice": (sphere_mesh((0.0, 0.0, 0.0), 0.16, 8, 16), 0.02, np.eye(3), np.zeros(3)),
    }


@pytest.mark.parametrize("name", ["box", "torus", "sphere", "sphere_on_lattice"])
def test_sample_solid_matches_cpu_restatement(name):
    from warpsph_b200.model import sample_solid

    (v, t), spacing, rot, pos = _meshes()[name]
    got = sample_solid(v, t, spacing, rot, pos)
    want = MO.sample_solid(v, t, spacing, rot, pos)
    assert len(want) > 100
    assert got.dtype == np.float32 and np.array_equal(got, want), (len(got), len(want))


def test_sample_solid_volume_and_shape():
    """The sampled torus lies within the tube (up to the facets' chord error)
    and its count matches the solid's volume to a few percent."""
    from warpsph_b200.model import sample_solid, torus_mesh

    v, t = torus_mesh((0, 0, 0), 0.3, 0.1, 96, 48)
    p = sample_solid(v, t, 0.01).astype(np.float64)
    r = np.hypot(p[:, 0], p[:, 2])
    d = np.hypot(r - 0.3, p[:, 1])
    assert d.max() <= 0.1 + 1e-6
    vol = 2 * np.pi ** 2 * 0.3 * 0.1 ** 2
    assert abs(len(p) * 0.01 ** 3 / vol - 1) < 0.03


def test_load_model_obj_round_trip(tmp_path, monkeypatch):
    """load_model (model.py:53-60) from an OBJ file: scale, lattice, rotation
    and translation as the reference applies them; the second call comes from
    the cache."""
    from warpsph_b200 import model

    monkeypatch.setattr(model, "CACHE_DIR", tmp_path / "cache")
    v, t = model.torus_mesh((0.0, 0.1, 0.0), 3.0, 1.0, 40, 20)
    path = tmp_path / "ring.obj"
    model.save_obj(path, v, t)
    pts = model.load_model(path, scale=0.1, pos=np.array([1.0, 2.0, 3.0]), rot=HAND_ROT, spacing=0.02)
    vv, tt = model.load_obj(path)
    want = MO.sample_solid(vv * 0.1, tt, 0.02, HAND_ROT, np.array([1.0, 2.0, 3.0]))
    assert np.array_equal(pts, want)
    assert len(list((tmp_path / "cache").glob("*.npz"))) == 1
    again = model.load_model(path, scale=0.1, pos=np.array([1.0, 2.0, 3.0]), rot=HAND_ROT, spacing=0.02)
    assert np.array_equal(again, pts)


def test_hand_scene_with_mesh_model(tmp_path, monkeypatch):
    """The reference's HAND scene recipe (IISPH.py:758-761, 976-984,
    1061-1081) on a smaller box: the model file's solid becomes rigid boundary
    particles after the box walls, moving at (0, 0.1, 0) m/s from the first
    step on."""
    import wp_sph.main as main
    from warpsph_b200 import model
    from warpsph_b200.solver import IISPH

    v, t = model.torus_mesh((0.0, 0.0, 0.0), 1.0, 0.4, 32, 16)
    monkeypatch.setattr(main, "MODEL_DIR", tmp_path)
    model.save_obj(tmp_path / "hand.obj", v, t)
    monkeypatch.setattr(model, "CACHE_DIR", tmp_path / "cache")
    monkeypatch.setattr(main, "scene_type", main.SceneType.HAND)
    monkeypatch.setattr(main, "DIAMETER", 0.05)
    monkeypatch.setattr(main, "GRAVITY", 9.8)
    monkeypatch.setattr(main, "BOX_WIDTH", 1.0)
    monkeypatch.setattr(main, "BOX_HEIGHT", 2.0)
    monkeypatch.setattr(main, "BOX_LENGTH", 1.0)
    monkeypatch.setitem(main.SCENE_MODELS, main.SceneType.HAND, [("hand.obj", 0.3, (0.5, 0.6, 0.5), np.eye(3))])
    sol = IISPH(stage_path=None)
    rigid = MO.sample_solid(v * 0.3, t, 0.05, np.eye(3), np.array([0.5, 0.6, 0.5]))
    assert sol.boundary_n == sol.boundary_hide_n + len(rigid)
    bx0 = sol.boundary_x.numpy()
    assert np.array_equal(bx0[sol.boundary_hide_n:], rigid)
    assert np.all(sol.boundary_v[sol.boundary_hide_n:] == np.float32([0.0, 0.1, 0.0]))
    for _ in range(5):
        sol.step()
    moved = sol.boundary_x.numpy()[sol.boundary_hide_n:] - rigid
    assert np.allclose(moved[:, 1], 0.1 * sol.sim_time, rtol=1e-3)
    assert np.all(moved[:, [0, 2]] == 0)
    assert np.array_equal(sol.boundary_x.numpy()[: sol.boundary_hide_n], bx0[: sol.boundary_hide_n])
    sol.close()
