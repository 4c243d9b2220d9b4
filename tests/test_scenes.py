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
