"""Emitters: appending fluid on the device (sph_add_fluid) keeps every existing
particle's state and equals building the grown state from scratch; a short pour
onto the procedural obstacle runs clean."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dam(n_side=12):
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import dam_break

    scene = dam_break(fluid=(n_side,) * 3, spacing=0.02, box=(0.6, 0.5, 0.4), jitter=1e-4, layers=2, seed=5)
    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024,
                          domain_min=(-0.06, -0.06, -0.06), domain_max=(0.66, 0.56, 0.46))
    return scene, params


def _new_layer(k, y=0.35):
    rng = np.random.default_rng(k)
    ix, iz = np.meshgrid(np.arange(8), np.arange(8), indexing="ij")
    x = np.stack([0.1 + ix.ravel() * 0.02, np.full(64, y), 0.1 + iz.ravel() * 0.02], axis=1)
    x = (x + rng.uniform(-1e-4, 1e-4, x.shape)).astype(np.float32)
    v = np.zeros_like(x)
    v[:, 1] = -1.0
    return x, v


def _new_block():
    """A 13 x 11 x 16 block at 0.02 m beside the dam's fluid."""
    rng = np.random.default_rng(9)
    g = np.meshgrid(np.arange(13), np.arange(11), np.arange(16), indexing="ij")
    x = np.stack([0.3 + g[0].ravel() * 0.02, 0.25 + g[1].ravel() * 0.02, 0.05 + g[2].ravel() * 0.02], axis=1)
    x = (x + rng.uniform(-1e-4, 1e-4, x.shape)).astype(np.float32)
    return x, np.zeros_like(x)


def test_add_fluid_equals_rebuilt_state():
    from warpsph_b200.solver import IISPH

    scene, params = _dam()
    a = IISPH(stage_path=None, params=params, scene=scene)
    a.steps(5)
    for k in range(3):  # the first and the third append outgrow the allocation
        xa, va, pa, dt = a.x.numpy(), a.v.numpy(), a.p.numpy(), a.dt
        xn, vn = _new_layer(k) if k < 2 else _new_block()
        a.add_fluid(xn, vn)
        assert a.n == len(xa) + len(xn)
        got = a.x.numpy()
        assert np.array_equal(got[: len(xa)], xa) and np.array_equal(got[len(xa):], xn)
        assert np.array_equal(a.p.numpy()[: len(xa)], pa) and not a.p.numpy()[len(xa):].any()
        b = IISPH(stage_path=None, params=params, scene=scene)
        b.set_state(np.concatenate([xa, xn]), np.concatenate([va, vn]))
        b.set_pressure(np.concatenate([pa, np.zeros(len(xn), np.float32)]))
        b.set_dt(dt)
        a.step()
        b.step()
        assert a.last_stats["iterations"] == b.last_stats["iterations"]
        for f in ("x", "v", "p", "rho"):
            assert np.array_equal(getattr(a, f).numpy(), getattr(b, f).numpy()), (k, f)
        b.close()
    a.close()


def test_short_pour_runs_clean():
    from warpsph_b200 import _lib, pour

    sol, inlet = pour.make(max_particles=12 * 1444, warm_start="zero")
    steps = pour.emit_until(sol, inlet)
    assert sol.n == 12 * 1444 and inlet.layers == 12
    assert 100 <= steps <= 130  # 11 more layers, one every 4 ms at dt = 4e-4 s
    sol.steps(20)
    h = sol.stats_history(20)
    assert not any(s["flags"] & (_lib.SPH_F_NONFINITE | _lib.SPH_F_TIMEOUT) for s in h)
    y = sol.x.numpy()[:, 1]
    assert y.max() < 1.8 + 1e-3 and y.min() > 0.0  # fell from the opening, still in the box
    v = sol.v.numpy()
    assert v[:, 1].mean() < -2.0  # accelerating downward
    sol.close()
