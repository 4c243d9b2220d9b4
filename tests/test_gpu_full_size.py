"""The benchmark's own workload at full size: the 1,000,000-particle dam break
(100 x 100 x 100 fluid lattice at 0.01 m, 206,464 boundary particles).

One step from a moving state, 30 steps after the start, against the FP32 CPU
oracle on the same inputs (the oracle finishes a full-size step in about a
second on the host's threads), and properties that hold at any size: the
neighbour relation is symmetric, the pair total the device counts equals the
exported lists, and the solve's reported average density error is exactly
what its exported terms give."""
import numpy as np
import pytest

from tests.helpers import csr_equal, elemstats, jacobi_output_ok, parity_floors

pytestmark = pytest.mark.gpu

RTOL = 1e-4
FIXED = 4  # fixed Jacobi iterations: both sides stop after the same update


@pytest.fixture(scope="module")
def full_step(oracle):
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.solver import IISPH
    from warpsph_b200.tables import kernel_tables

    params = preset_params("dam_break_1m", keep_fb_lists=True)
    scene = preset_scene("dam_break_1m")
    run = IISPH(stage_path=None, params=params, scene=scene)
    run.steps(30)
    x, v, dt = run.x.numpy(), run.v.numpy(), run.dt
    psi = run.boundary_phi.numpy()
    run.close()

    sol = IISPH(stage_path=None, params=params.replace(fixed_iters=FIXED), scene=scene)
    sol.set_state(x, v)
    sol.set_dt(dt, 1.0 / dt)
    sol.step()
    out = {"stats": dict(sol.last_stats), "nb": sol.get_neighbors(with_boundary=True),
           "rho": sol.rho.numpy(), "rho_adv": sol.rho_adv.numpy(), "a_ii": sol.term_a_ii.numpy(),
           "Ap": sol.term_Ap_i.numpy(), "p": sol.p.numpy(), "v": sol.v.numpy(), "x": sol.x.numpy()}
    sol.close()

    op = oracle.reference_params(diameter=params.diameter, gravity=params.gravity, w_size=params.w_table_size,
                                 g_size=params.g_table_size)
    ref = oracle.step(op, x, v, scene.boundary_x, None, psi, dt, 1.0 / dt, tables=kernel_tables(params),
                      fixed_iters=FIXED)
    truth = oracle.step(op, x, v, scene.boundary_x, None, psi, dt, 1.0 / dt, tables=oracle.kernel_tables(op, np.float64),
                        precision="f64", fixed_iters=FIXED)
    out["dt"] = dt
    return out, (ref, truth), params


def test_full_size_step_vs_oracle(full_step):
    """Per element (tests.helpers): the terms before the solve within 1e-4 of
    the FP32 oracle, p and v within 1e-4 or at the FP32 noise floor against
    the FP64 oracle, x within 1e-4 of the spacing."""
    out, (ref, truth), params = full_step
    fl = parity_floors(params, out["dt"])
    assert out["stats"]["iterations"] == FIXED
    assert csr_equal(out["nb"]["ff_off"], out["nb"]["ff_idx"], ref["ff_off"], ref["ff_idx"])
    assert csr_equal(out["nb"]["fb_off"], out["nb"]["fb_idx"], ref["fb_off"], ref["fb_idx"])
    for k in ("rho", "rho_adv", "a_ii"):
        assert elemstats(out[k], ref[k], fl[k])[0] < RTOL, k
    for k in ("p", "v"):
        ok, detail = jacobi_output_ok(out[k], ref[k], truth[k], fl[k])
        assert ok, (k, detail)
    assert elemstats(out["x"], ref["x"], fl["x"], x_like=True)[0] < RTOL


def test_full_size_neighbour_relation_symmetric(full_step):
    out, _, _ = full_step
    off = np.asarray(out["nb"]["ff_off"], np.int64)
    idx = np.asarray(out["nb"]["ff_idx"], np.int64)
    n = len(off) - 1
    assert out["stats"]["n_ff_pairs"] == len(idx)
    i = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    assert not np.any(i == idx)  # no particle lists itself
    fwd = np.sort(i * n + idx)
    bwd = np.sort(idx * n + i)
    assert np.array_equal(fwd, bwd)


def test_full_size_reported_error_matches_terms(full_step):
    """update_rho_error + average_rho_error (IISPH.py:542-568, 1489-1494):
    per particle in FP32, summed in FP64; only the summation order differs."""
    out, _, params = full_step
    rho0 = np.float32(params.rho0)
    rp = (out["rho_adv"] + out["Ap"]).astype(np.float32)
    hot = rp > rho0
    err = np.abs(rp[hot] / rho0 - np.float32(1.0)).astype(np.float32)
    want = float(np.sum(err.astype(np.float64)) / max(int(hot.sum()), 1))
    assert abs(out["stats"]["avg_err"] - want) <= 1e-12 * max(want, 1e-30)
    assert np.all(np.isfinite(out["x"])) and np.all(np.isfinite(out["v"])) and np.all(out["p"] >= 0)


def test_full_size_runs_repeat_bit_for_bit():
    """Two runs of the same 1M steps give the same words: the sort's order
    is a function of the positions, every sum runs in list order, and the
    solve's FP64 residual adds per-block partials in block order, so the
    iteration counts and every state word repeat whatever the scheduling
    (learned start with continuation, steps [0, 12), which include capped
    solves)."""
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.solver import IISPH

    scene = preset_scene("dam_break_1m")
    runs = []
    for _ in range(2):
        params = preset_params("dam_break_1m", warm_start="mlp", warm_continue=True)
        sol = IISPH(stage_path=None, params=params, scene=scene)
        sol.steps(12)
        hist = [(h["iterations"], h["avg_err"]) for h in sol.stats_history(12)]
        runs.append((hist, sol.x.numpy(), sol.v.numpy(), sol.p.numpy()))
        sol.close()
    assert runs[0][0] == runs[1][0]
    for a, b in zip(runs[0][1:], runs[1][1:]):
        assert np.array_equal(a, b)


def test_full_size_batch_of_64_matches_individual_runs():
    """The batched workload at full size: 64 dam breaks of 5k-200k particles
    (log-uniform, seeded) in one context with the learned warm start, against
    the smallest, the median and the largest scene run alone, bit for bit."""
    from warpsph_b200.batch import BatchIISPH
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import batched_scenes
    from warpsph_b200.solver import IISPH

    scenes = batched_scenes()
    assert len(scenes) == 64
    params = SolverParams(diameter=0.01, gravity=9.81, w_table_size=1024, g_table_size=1024, warm_start="mlp")
    steps = 20
    b = BatchIISPH(scenes, params)
    b.steps(steps)
    st = b.scene_stats()
    order = np.argsort([s.n for s in scenes])
    for k in (int(order[0]), int(order[len(order) // 2]), int(order[-1])):
        sol = IISPH(stage_path=None, params=params, scene=scenes[k])
        sol.steps(steps)
        x, v, p = b.scene_fluid(k)
        assert np.array_equal(x, sol.x.numpy()), k
        assert np.array_equal(v, sol.v.numpy()), k
        assert np.array_equal(p, sol.p.numpy()), k
        assert st["iterations"][k] == sol.last_stats["iterations"], k
        sol.close()
    b.close()


def test_full_size_pour_step_vs_oracle(oracle):
    """The pour at full size: 2,000,000 particles emitted layer by layer onto
    the seeded obstacle union (about 1M boundary particles), then one step of
    the filled scene against the oracle: uneven cell occupancy, splashes and
    particles resting on curved boundaries."""
    from warpsph_b200 import _lib, pour
    from warpsph_b200.params import POUR
    from warpsph_b200.tables import kernel_tables

    sol, inlet = pour.make(warm_start="zero", keep_fb_lists=True)
    pour.emit_until(sol, inlet)
    assert sol.n == POUR["max_particles"]
    sol.steps(5)
    hist = sol.stats_history(5)
    assert not any(h["flags"] & (_lib.SPH_F_NONFINITE | _lib.SPH_F_TIMEOUT) for h in hist)
    x, v, dt = sol.x.numpy(), sol.v.numpy(), sol.dt
    psi = sol.boundary_phi.numpy()
    bx = sol.boundary_x.numpy()
    params = sol.params
    sol.close()

    one, _ = pour.make(warm_start="zero", keep_fb_lists=True, fixed_iters=FIXED)
    one.set_state(x, v)
    one.set_dt(dt, 1.0 / dt)
    one.step()
    nb = one.get_neighbors(with_boundary=True)
    op = oracle.reference_params(diameter=params.diameter, gravity=params.gravity, w_size=params.w_table_size,
                                 g_size=params.g_table_size)
    ref = oracle.step(op, x, v, bx, None, psi, dt, 1.0 / dt, tables=kernel_tables(params), fixed_iters=FIXED)
    truth = oracle.step(op, x, v, bx, None, psi, dt, 1.0 / dt, tables=oracle.kernel_tables(op, np.float64),
                        precision="f64", fixed_iters=FIXED)
    fl = parity_floors(params, dt)
    assert one.last_stats["iterations"] == FIXED
    assert csr_equal(nb["ff_off"], nb["ff_idx"], ref["ff_off"], ref["ff_idx"])
    assert csr_equal(nb["fb_off"], nb["fb_idx"], ref["fb_off"], ref["fb_idx"])
    for k, got in (("rho", one.rho), ("rho_adv", one.rho_adv)):
        assert elemstats(got.numpy(), ref[k], fl[k])[0] < RTOL, k
    for k, got in (("p", one.p), ("v", one.v)):
        ok, detail = jacobi_output_ok(got.numpy(), ref[k], truth[k], fl[k])
        assert ok, (k, detail)
    assert elemstats(one.x.numpy(), ref["x"], fl["x"], x_like=True)[0] < RTOL
    one.close()
