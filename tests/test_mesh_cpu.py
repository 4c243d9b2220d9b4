"""Mesh models on the CPU: the OBJ reader and the sampler's CPU restatement
(oracle/mesh_oracle.py) against analytic solids."""
import numpy as np

from oracle import mesh_oracle as MO
from warpsph_b200.model import box_mesh, load_obj, save_obj, sphere_mesh, torus_mesh


def test_obj_reader_polygons_and_index_forms(tmp_path):
    p = tmp_path / "q.obj"
    p.write_text("# a quad and a triangle\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\n"
                 "f 1/1/1 2/2/1 3/3/1 4/4/1\nv 0 0 1\nf -1 1 2\n")
    v, t = load_obj(p)
    assert v.shape == (5, 3)
    assert t.tolist() == [[0, 1, 2], [0, 2, 3], [4, 0, 1]]


def test_obj_round_trip(tmp_path):
    v, t = torus_mesh((0.1, 0.2, 0.3), 0.5, 0.2, 12, 6)
    save_obj(tmp_path / "t.obj", v, t)
    v2, t2 = load_obj(tmp_path / "t.obj")
    assert np.array_equal(v, v2) and np.array_equal(t, t2)


def test_box_lattice_is_all_inside():
    """Every lattice point of a box's own lattice is inside: the lattice
    starts on the faces +x enters through and stops short of the others."""
    v, t = box_mesh((0.1, 0.2, 0.3), (0.5, 0.45, 0.7))
    p = MO.sample_solid(v, t, 0.02)
    n = np.prod([len(np.arange(v.min(0)[a], v.max(0)[a], 0.02)) for a in range(3)])
    assert len(p) == n


def test_sphere_and_torus_volumes():
    v, t = sphere_mesh((0.0, 0.0, 0.0), 0.2, 24, 48)
    p = MO.sample_solid(v, t, 0.01)
    assert np.linalg.norm(p, axis=1).max() <= 0.2 + 1e-6
    assert abs(len(p) * 1e-6 / (4 / 3 * np.pi * 0.2 ** 3) - 1) < 0.03
    v, t = torus_mesh((0.0, 0.0, 0.0), 0.3, 0.1, 64, 32, axis="z")
    p = MO.sample_solid(v, t, 0.01).astype(np.float64)
    d = np.hypot(np.hypot(p[:, 0], p[:, 1]) - 0.3, p[:, 2])
    assert d.max() <= 0.1 + 1e-6
