"""Batched scenes: one launch sequence per step for many independent scenes
must reproduce each scene's own run exactly (same grid, sorted order, chunk
partition and per-scene convergence decisions)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenes():
    from warpsph_b200.scenes import dam_break

    return [dam_break(fluid=(12, 10, 8), spacing=0.02, box=(0.5, 0.4, 0.2), jitter=1e-4, seed=1),
            dam_break(fluid=(6, 14, 6), spacing=0.02, box=(0.3, 0.5, 0.2), jitter=1e-4, seed=2),
            dam_break(fluid=(20, 8, 10), spacing=0.02, box=(0.8, 0.3, 0.3), jitter=1e-4, seed=3,
                      velocity=(0.0, -0.4, 0.0)),
            dam_break(fluid=(3, 3, 3), spacing=0.02, box=(0.2, 0.2, 0.2), jitter=1e-4, seed=4)]


@pytest.mark.parametrize("warm", ["zero", "half", "mlp_continue"])
def test_batch_matches_individual_runs(warm):
    """With "mlp_continue" the iteration cap is low, so some scenes' solves
    stop at it and continue from their own pressure while the others start
    from the network's prediction."""
    from warpsph_b200.batch import BatchIISPH
    from warpsph_b200.params import SolverParams
    from warpsph_b200.solver import IISPH

    kw = dict(warm_start="mlp", warm_continue=True, max_loop=8) if warm == "mlp_continue" else dict(warm_start=warm)
    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024, **kw)
    scenes = _scenes()
    b = BatchIISPH(scenes, params)
    steps = 40
    b.steps(steps)
    st = b.scene_stats()
    capped = []
    for k, sc in enumerate(scenes):
        sol = IISPH(stage_path=None, params=params, scene=sc)
        sol.steps(steps)
        capped.append(sum(h["iterations"] == params.max_loop + 1 for h in sol.stats_history(steps)))
        x, v, p = b.scene_fluid(k)
        assert np.array_equal(x, sol.x.numpy()), k
        assert np.array_equal(v, sol.v.numpy()), k
        assert np.array_equal(p, sol.p.numpy()), k
        assert st["iterations"][k] == sol.last_stats["iterations"], k
        assert st["sim_time"][k] == sol.sim_time, k
        sol.close()
    b.close()
    if warm == "mlp_continue":
        assert sum(capped) > 0, capped


def test_batch_scene_ranges_and_empty_scene():
    from warpsph_b200.batch import BatchIISPH
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import Scene, dam_break

    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024)
    a = dam_break(fluid=(8, 8, 8), spacing=0.02, box=(0.3, 0.3, 0.3), jitter=1e-4, seed=5)
    empty = Scene(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), a.boundary_x.copy(), len(a.boundary_x),
                  a.box)
    b = BatchIISPH([a, empty, a], params)
    assert list(b.fluid_off) == [0, a.n, a.n, 2 * a.n]
    b.steps(5)
    st = b.scene_stats()
    assert st["iterations"][1] == 2 and st["avg_err"][1] == 0.0
    x0, _, _ = b.scene_fluid(0)
    x2, _, _ = b.scene_fluid(2)
    assert np.array_equal(x0, x2)  # identical scenes evolve identically
    b.close()


def test_launch_shapes_do_not_change_results():
    """Every solve shape the autotuner may pick gives the same trajectory."""
    from warpsph_b200.autotune import SOLVE_SHAPES
    from warpsph_b200.batch import BatchIISPH
    from warpsph_b200.params import SolverParams

    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024)
    scenes = _scenes()
    ref = None
    for blk, ppt, unr in SOLVE_SHAPES[::2] + [SOLVE_SHAPES[-1]]:
        b = BatchIISPH(scenes, params.replace(block_size=64, jacobi_block=blk, jacobi_ppt=ppt, jacobi_unroll=unr))
        b.steps(15)
        out = b.fluid()
        b.close()
        if ref is None:
            ref = out
        else:
            for u, w in zip(out, ref):
                np.testing.assert_allclose(u, w, rtol=1e-5, atol=1e-7)


def test_autotune_returns_valid_shape(tmp_path, monkeypatch):
    import warpsph_b200.autotune as at
    from warpsph_b200.params import SolverParams

    monkeypatch.setattr(at, "CACHE", tmp_path / "tune.json")
    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024)
    res = at.autotune(_scenes(), params, warm=3, steps=5)
    assert res["block_size"] in at.BUILD_BLOCKS
    assert (res["jacobi_block"], res["jacobi_ppt"], res["jacobi_unroll"]) in at.SOLVE_SHAPES
    assert isinstance(res["plain_loads"], bool)
    again = at.autotune(_scenes(), params, warm=3, steps=5)
    assert again == res  # served from the cache
