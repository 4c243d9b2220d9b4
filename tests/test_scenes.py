"""Scene construction: the vectorised init_particles reproduces the reference's
loop-built particle sets and order (IISPH.py:857-1000).  No GPU needed."""
import numpy as np

from warpsph_b200.scenes import box_scene, dam_break, reference_empty_scene


def init_particles_loops(box, spacing, min_point, max_point, fluid_depth=0.0, boundary_layers=3):
    """Literal restatement of the reference's Python loops, for small boxes."""
    bw, bh, bl = box
    xr = range(-boundary_layers, int(bw / spacing) + boundary_layers)
    yr = range(-boundary_layers, int(bh / spacing) + boundary_layers)
    zr = range(-boundary_layers, int(bl / spacing) + boundary_layers)
    x_max, y_max, z_max = int(bw / spacing) - 1, int(bh / spacing) - 1, int(bl / spacing) - 1
    boundary, fluid = [], []
    fluid_y_max = int(fluid_depth / spacing) if fluid_depth > 0 else -1
    for xi in xr:
        for yi in yr:
            for zi in zr:
                x, y, z = xi * spacing, yi * spacing, zi * spacing
                outside = xi < 0 or xi > x_max or yi < 0 or yi > y_max or zi < 0 or zi > z_max
                if outside:
                    boundary.append([x, y, z])
                elif fluid_depth > 0 and yi <= fluid_y_max:
                    in_rect = (min_point[0] - spacing < x < max_point[0] + spacing
                               and min_point[1] - spacing < y < max_point[1] + spacing
                               and min_point[2] - spacing < z < max_point[2] + spacing)
                    if not in_rect:
                        fluid.append([x, y, z])
    xs = np.arange(min_point[0], max_point[0], spacing)
    ys = np.arange(min_point[1], max_point[1], spacing)
    zs = np.arange(min_point[2], max_point[2], spacing)
    xx, yy, zz = np.meshgrid(xs, ys, zs, indexing="ij")
    fluid.extend(np.stack([xx.ravel(), yy.ravel(), zz.ravel()]).T)
    return np.array(boundary, np.float32), np.array(fluid, np.float32)


def test_box_scene_matches_loops():
    box, sp = (0.6, 0.45, 0.35), 0.05
    mn, mx = (0.1, 0.05, 0.05), (0.4, 0.3, 0.2)
    for depth in (0.0, 0.12):
        b, f = init_particles_loops(box, sp, mn, mx, fluid_depth=depth)
        s = box_scene(box, sp, mn, mx, fluid_depth=depth)
        assert np.array_equal(s.boundary_x, b)
        assert np.array_equal(s.fluid_x, f)


def test_reference_default_scene_counts():
    s = reference_empty_scene()
    assert (s.n, s.boundary_n) == (102641, 124056)


def test_dam_break_presets():
    s = dam_break(fluid=(20, 20, 20), spacing=0.02, box=(1.0, 0.6, 0.4), jitter=1e-4, layers=2, seed=0)
    assert s.n == 8000 and s.boundary_n == 14064
    lattice = dam_break(fluid=(20, 20, 20), spacing=0.02, box=(1.0, 0.6, 0.4), jitter=0.0, layers=2)
    dev = np.abs(s.fluid_x.astype(np.float64) - lattice.fluid_x)
    assert dev.max() <= 1e-4 + 1e-7 and dev.max() > 5e-5
    big = dam_break(fluid=(4, 4, 4), spacing=0.01, box=(2.0, 1.0, 1.0), jitter=5e-5, layers=2, seed=1)
    assert big.boundary_n == 206464


def test_pour_obstacle_union_surface():
    """The obstacle union is seeded and keeps no particle strictly inside
    another shape of the union."""
    from warpsph_b200.scenes import _inside_box, _inside_torus, pour_obstacles

    a, shapes = pour_obstacles(seed=2, spacing=0.008)
    b, _ = pour_obstacles(seed=2, spacing=0.008)
    assert np.array_equal(a, b) and len(a) > 20000
    assert len(shapes) == 10 and sum(s[0] == "box" for s in shapes) == 6
    for sh in shapes:
        inside = (_inside_box(a, sh[1], sh[2], 0.5 * 0.008) if sh[0] == "box"
                  else _inside_torus(a, sh[1], sh[2], sh[3], sh[4], 0.5 * 0.008))
        assert not inside.any()
    for sh in shapes:
        if sh[0] == "box":
            half = (np.asarray(sh[2]) - np.asarray(sh[1])) / 2
            assert np.all(half >= 0.05 - 1e-9) and np.all(half <= 0.2 + 1e-9)
        else:
            assert 0.05 <= sh[2] <= 0.2


def test_inlet_schedule():
    """Layer k leaves the opening at k * spacing / speed and sits (t - t_k) * speed
    below it at time t; emission stops at max_particles."""
    from warpsph_b200.scenes import Inlet

    inl = Inlet(center=(1.0, 1.8, 1.0), size=(0.3, 0.3), spacing=0.008, speed=2.0, max_particles=5000, jitter=0.0)
    assert inl.layer_size == 38 * 38 and abs(inl.period - 0.004) < 1e-15
    x, v = inl.due(0.0)
    assert len(x) == inl.layer_size and np.allclose(x[:, 1], 1.8) and np.allclose(v[:, 1], -2.0)
    x, v = inl.due(0.0101)  # layers 1 and 2 (t = 0.004, 0.008)
    assert len(x) == 2 * inl.layer_size
    ys = np.unique(np.round(x[:, 1], 5))
    assert np.allclose(sorted(ys), [1.8 - 0.0061 * 2, 1.8 - 0.0021 * 2], atol=1e-5)
    x, _ = inl.due(1.0)
    assert inl.emitted == 5000 and inl.done and len(x) == 5000 - 3 * inl.layer_size
    assert len(inl.due(2.0)[0]) == 0
    xs = x[:, [0, 2]]
    assert xs.min() > 1.0 - 0.15 - 1e-6 and xs.max() < 1.0 + 0.15 + 1e-6


def test_pour_scene_counts():
    from warpsph_b200.scenes import pour_scene

    sc, inlet = pour_scene()
    assert sc.boundary_hide_n == 762064           # 2 wall layers of the 2 m cube at 0.008 m
    assert sc.boundary_n > sc.boundary_hide_n + 20000
    assert sc.n == inlet.layer_size and inlet.layers == 1
