"""GPU parity: libwpsph (through its C ABI, via the drop-in IISPH class) against
the reference's golden vectors and the CPU oracle on identical input states.

Bars (from the hot-path contract):
  * neighbour sets bit-exact (integer work);
  * per-step density, pressure, positions within 1e-4 relative, per element
    (tests.helpers.elemrel with the floors of tests.helpers.parity_floors);
  * Jacobi iteration count within +-1; p, s, v and x are always compared at
    the reference's iteration count (a twin context with fixed iterations
    where the counts differ).
"""
import numpy as np
import pytest

from tests.helpers import (csr_equal, elemstats, golden_oracle_params, golden_solver_params, jacobi_output_ok,
                           load_golden, normrel, parity_floors)

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def assert_elem(got, want, floor, what, bar=RTOL, x_like=False):
    mx, p999 = elemstats(got, want, floor, x_like)
    assert mx < bar, f"{what}: per-element max {mx:.3g} (p99.9 {p999:.3g}) over {bar}"


def assert_jacobi(got, want, truth, floor, what):
    ok, detail = jacobi_output_ok(got, want, truth, floor)
    assert ok, f"{what}: {detail}"


def _golden_truth(oracle, G, meta, s, iterations):
    """FP64 oracle of golden step s at the reference's iteration count."""
    P = golden_oracle_params(oracle, meta)
    pre = f"s{s}_"
    return oracle.step(P, G[pre + "x_in"], G[pre + "v_in"], G["boundary_x"], None, G["boundary_phi"],
                       float(G[pre + "dt_in"]), float(G[pre + "inv_dt_in"]),
                       tables=oracle.kernel_tables(P, np.float64), precision="f64", fixed_iters=iterations)


def _solver(params, scene):
    from warpsph_b200.solver import IISPH

    return IISPH(stage_path=None, params=params, scene=scene)


def _golden_params(meta, **kw):
    return golden_solver_params(meta, keep_fb_lists=True, **kw)


def _golden_scene(G, s):
    from warpsph_b200.scenes import Scene

    bx = G["boundary_x"]
    return Scene(G[f"s{s}_x_in"], G[f"s{s}_v_in"], bx, len(bx), (0, 0, 0))


@pytest.mark.parametrize("name", ["ref_lattice", "dam_jitter", "compressed", "viscous"])
def test_golden_steps(oracle, name):
    G, meta = load_golden(name)
    params = _golden_params(meta)
    sol = _solver(params, _golden_scene(G, 0))
    assert_elem(sol.boundary_phi.numpy(), G["boundary_phi"], 0.0, "psi", bar=1e-5)
    for s in range(int(G["steps"])):
        pre = f"s{s}_"
        dt = float(G[pre + "dt_in"])
        fl = parity_floors(params, dt)
        sol.set_state(G[pre + "x_in"], G[pre + "v_in"])
        sol.set_dt(dt, float(G[pre + "inv_dt_in"]))
        sol.step()
        nb = sol.get_neighbors(with_boundary=True)
        assert csr_equal(nb["ff_off"], nb["ff_idx"], G[pre + "ff_off"], G[pre + "ff_idx"]), f"ff sets, step {s}"
        assert csr_equal(nb["fb_off"], nb["fb_idx"], G[pre + "fb_off"], G[pre + "fb_idx"]), f"fb sets, step {s}"
        for q, got in (("rho", sol.rho), ("rho_adv", sol.rho_adv), ("v_adv", sol.v_adv), ("d_ii", sol.term_d_ii),
                       ("a_ii", sol.term_a_ii)):
            assert_elem(got.numpy(), G[pre + q], fl[q], f"{q}, step {s}")
        it_ref = int(G[pre + "iterations"])
        it = sol.last_stats["iterations"]
        assert abs(it - it_ref) <= 1, (it, it_ref)
        src = sol
        if it != it_ref:
            # the reference's iteration count from the same inputs
            src = _solver(params.replace(fixed_iters=it_ref), _golden_scene(G, s))
            src.set_dt(dt, float(G[pre + "inv_dt_in"]))
            src.step()
            assert src.last_stats["iterations"] == it_ref
        truth = _golden_truth(oracle, G, meta, s, it_ref)
        assert_jacobi(src.p.numpy(), G[pre + "p"], truth["p"], fl["p"], f"p, step {s}")
        assert_jacobi(src.sum_d_ij_p_j.numpy(), G[pre + "s"], truth["s"], fl["s"], f"s, step {s}")
        assert_elem(src.v.numpy(), G[pre + "v_out"], fl["v"], f"v, step {s}")
        assert_elem(src.x.numpy(), G[pre + "x_out"], fl["x"], f"x, step {s}", x_like=True)
        if src is not sol:
            src.close()
        assert abs(sol.dt - float(G[pre + "dt_out"])) <= 1e-4 * float(G[pre + "dt_out"])
    sol.close()


@pytest.mark.parametrize("name", ["dam_jitter", "compressed", "viscous"])
def test_golden_fixed_iterations(oracle, name):
    """Pressure after exactly the reference's iteration count, even where the
    convergence test would stop one iteration apart."""
    G, meta = load_golden(name)
    for s in range(int(G["steps"])):
        pre = f"s{s}_"
        sol = _solver(_golden_params(meta, fixed_iters=int(G[pre + "iterations"])), _golden_scene(G, s))
        sol.set_dt(float(G[pre + "dt_in"]), float(G[pre + "inv_dt_in"]))
        sol.step()
        assert sol.last_stats["iterations"] == int(G[pre + "iterations"])
        fl = parity_floors(sol.params, float(G[pre + "dt_in"]))
        truth = _golden_truth(oracle, G, meta, s, int(G[pre + "iterations"]))
        assert_jacobi(sol.p.numpy(), G[pre + "p"], truth["p"], fl["p"], f"p, step {s}")
        assert_jacobi(sol.term_Ap_i.numpy(), G[pre + "Ap"], truth["Ap"], fl["Ap"], f"Ap, step {s}")
        assert_elem(sol.v.numpy(), G[pre + "v_out"], fl["v"], f"v, step {s}")
        sol.close()


def _oracle_step(oracle, params, x, v, bx, psi, dt, inv_dt, precision="f32", tables=None, **kw):
    from warpsph_b200.tables import kernel_tables

    op = oracle.reference_params(diameter=params.diameter, gravity=params.gravity, w_size=params.w_table_size,
                                 g_size=params.g_table_size, vis_mu_scale=params.vis_mu_scale)
    tabs = kernel_tables(params) if tables is None else tables
    if precision == "f64":
        tabs = oracle.kernel_tables(op, np.float64) if tables is None else tuple(np.float64(t) for t in tables)
    return oracle.step(op, x, v, bx, None, psi, dt, inv_dt, tables=tabs, precision=precision, **kw)


_FIELDS = {"rho": "rho", "rho_adv": "rho_adv", "v_adv": "v_adv", "d_ii": "term_d_ii", "a_ii": "term_a_ii",
           "s": "sum_d_ij_p_j", "Ap": "term_Ap_i", "p": "p", "v": "v", "x": "x"}
_JACOBI = ("p", "s", "Ap", "v")


def assert_matches_oracle(oracle, sol, params, inputs, ref, keys, tables=None, **kw):
    """Per-element checks of sol's last step against the FP32 oracle step
    ``ref`` from ``inputs`` = (x, v, bx, psi, dt): 1e-4 for the terms before
    the solve and for x (in units of the spacing), the FP32 noise rule against
    an FP64 oracle step at the same iteration count for the Jacobi outputs."""
    x, v, bx, psi, dt = inputs
    fl = parity_floors(params, dt)
    truth = None
    for k in keys:
        got = getattr(sol, _FIELDS[k]).numpy()
        if k in _JACOBI:
            if truth is None:
                truth = _oracle_step(oracle, params, x, v, bx, psi, dt, 1.0 / dt, precision="f64", tables=tables,
                                     **dict(kw, fixed_iters=int(ref["iterations"])))
            assert_jacobi(got, ref[k], truth[k], fl[k], k)
        else:
            assert_elem(got, ref[k], fl[k], k, x_like=(k == "x"))


def _at_reference_count(sol, params, scene, x, v, dt, ref, pressure=None):
    """sol itself when its last step ran the reference's iteration count,
    else a twin context stepped from the same inputs with that many fixed
    iterations (the caller closes it if it is not sol)."""
    if sol.last_stats["iterations"] == int(ref["iterations"]):
        return sol
    twin = _solver(params.replace(fixed_iters=int(ref["iterations"])), scene)
    twin.set_state(x, v)
    if pressure is not None:
        twin.set_pressure(pressure)
    twin.set_dt(dt, 1.0 / dt)
    twin.step()
    assert twin.last_stats["iterations"] == int(ref["iterations"])
    return twin


def test_dam_break_8k_vs_oracle(oracle):
    """The 8,000-particle dam break: one step from the initial state and one
    from a state 30 GPU steps later, GPU vs the FP32 oracle (and FP64 truth)."""
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    params = preset_params("dam_break_8k", keep_fb_lists=True)
    scene = preset_scene("dam_break_8k")
    sol = _solver(params, scene)
    psi = sol.boundary_phi.numpy()
    op = oracle.reference_params(diameter=params.diameter, gravity=params.gravity, w_size=1024, g_size=1024)
    from warpsph_b200.tables import kernel_tables

    assert_elem(psi, oracle.boundary_psi(op, scene.boundary_x, tables=kernel_tables(params)), 0.0, "psi", bar=1e-5)
    for warm in (0, 30):
        if warm:
            sol.steps(warm)
        x, v = sol.x.numpy(), sol.v.numpy()
        dt = sol.dt
        ref = _oracle_step(oracle, params, x, v, scene.boundary_x, psi, dt, 1.0 / dt)
        sol.set_state(x, v)
        sol.set_dt(dt, 1.0 / dt)
        sol.step()
        nb = sol.get_neighbors(with_boundary=True)
        assert csr_equal(nb["ff_off"], nb["ff_idx"], ref["ff_off"], ref["ff_idx"])
        assert csr_equal(nb["fb_off"], nb["fb_idx"], ref["fb_off"], ref["fb_idx"])
        inputs = (x, v, scene.boundary_x, psi, dt)
        assert_matches_oracle(oracle, sol, params, inputs, ref, ("rho", "rho_adv", "d_ii", "a_ii"))
        assert abs(sol.last_stats["iterations"] - ref["iterations"]) <= 1
        src = _at_reference_count(sol, params, scene, x, v, dt, ref)
        assert_matches_oracle(oracle, src, params, inputs, ref, ("p", "s", "v", "x"))
        if src is not sol:
            src.close()
    sol.close()


def test_viscous_dam_break_vs_oracle(oracle):
    """Viscosity on (VIS_MU = 0.01 RHO_0): the three-pass build (lists and rho,
    v_adv with the laplacian, advection terms) on the 8,000-particle dam break
    after 40 steps of flow, one step against the FP32 oracle."""
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    params = preset_params("dam_break_8k", keep_fb_lists=True, vis_mu_scale=0.01)
    scene = preset_scene("dam_break_8k")
    sol = _solver(params, scene)
    psi = sol.boundary_phi.numpy()
    sol.steps(40)
    x, v = sol.x.numpy(), sol.v.numpy()
    dt = sol.dt
    ref = _oracle_step(oracle, params, x, v, scene.boundary_x, psi, dt, 1.0 / dt)
    sol.set_state(x, v)
    sol.set_dt(dt, 1.0 / dt)
    sol.step()
    nb = sol.get_neighbors(with_boundary=True)
    assert csr_equal(nb["ff_off"], nb["ff_idx"], ref["ff_off"], ref["ff_idx"])
    inputs = (x, v, scene.boundary_x, psi, dt)
    assert_matches_oracle(oracle, sol, params, inputs, ref, ("rho", "v_adv", "rho_adv", "a_ii"))
    assert abs(sol.last_stats["iterations"] - ref["iterations"]) <= 1
    src = _at_reference_count(sol, params, scene, x, v, dt, ref)
    assert_matches_oracle(oracle, src, params, inputs, ref, ("p", "v", "x"))
    if src is not sol:
        src.close()
    # the viscous term is really on: v_adv differs from v - g dt y
    base = v.copy()
    base[:, 1] -= params.gravity * dt
    assert np.abs(sol.v_adv.numpy() - base).max() > 1e-3
    sol.close()


@pytest.mark.parametrize("g_size", [1024, 65536])
def test_table_gradient_path(oracle, g_size):
    """Gradient tables that are not the cubic spline's own samples (here one
    sample nudged) make the solve interpolate the table, staged in shared
    memory (1024 samples) or read from global memory (65536), instead of using
    the closed form; both agree with the oracle run on the same tables."""
    from warpsph_b200 import _lib
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.tables import kernel_tables

    params = preset_params("dam_break_8k", g_table_size=g_size, fixed_iters=6)
    scene = preset_scene("dam_break_8k")
    warm = _solver(params.replace(fixed_iters=-1), scene)
    warm.steps(20)
    x, v, psi, dt = warm.x.numpy(), warm.v.numpy(), warm.boundary_phi.numpy(), warm.dt
    warm.close()
    w, g = kernel_tables(params)
    g = g.copy()
    g[-1] = np.nextafter(np.float32(0), np.float32(1))  # was exactly 0 at r = h
    sol = _solver(params, scene)
    _lib.check(sol._ctx, sol._lib.sph_set_tables(sol._ctx, _lib.ptr(w), len(w), _lib.ptr(g), len(g)))
    sol.set_state(x, v)
    sol.set_dt(dt, 1.0 / dt)
    sol.step()
    op = oracle.reference_params(diameter=params.diameter, gravity=params.gravity, w_size=params.w_table_size,
                                 g_size=g_size)
    ref = oracle.step(op, x, v, scene.boundary_x, None, psi, dt, 1.0 / dt, tables=(w, g), fixed_iters=6)
    assert sol.last_stats["iterations"] == 6
    assert_matches_oracle(oracle, sol, params, (x, v, scene.boundary_x, psi, dt), ref, ("a_ii", "p", "Ap", "v"),
                          tables=(w, g))
    sol.close()


def test_warm_start_half_vs_oracle(oracle):
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    params = preset_params("dam_break_8k", warm_start="half")
    scene = preset_scene("dam_break_8k")
    sol = _solver(params, scene)
    sol.steps(20)
    x, v, p = sol.x.numpy(), sol.v.numpy(), sol.p.numpy()
    psi = sol.boundary_phi.numpy()
    ref = _oracle_step(oracle, params, x, v, scene.boundary_x, psi, sol.dt, 1.0 / sol.dt, p=p, warm_start=1,
                       fixed_iters=4)
    sol2 = _solver(params.replace(fixed_iters=4), scene)
    sol2.set_state(x, v)
    sol2.set_pressure(p)
    sol2.set_dt(sol.dt, 1.0 / sol.dt)
    sol2.step()
    assert_matches_oracle(oracle, sol2, params, (x, v, scene.boundary_x, psi, sol.dt), ref, ("p", "v", "x"),
                          p=p, warm_start=1)
    sol.close()
    sol2.close()


def test_warm_continue_after_capped_solve_vs_oracle(oracle):
    """Learned warm start with warm_continue: a solve that stopped at the
    iteration cap hands its final pressure to the next step as that step's
    first iterate, in place of the network's prediction.  The oracle's
    "keep p" start (Ap of the given p, then Jacobi updates) with one update
    fewer than the capped count is the same sequence of iterates."""
    from warpsph_b200 import _lib
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    max_loop = 3  # caps at 4 iterations: the dam break's first steps need ~100
    scene = preset_scene("dam_break_8k")
    params = preset_params("dam_break_8k", warm_start="mlp", warm_continue=True, max_loop=max_loop)
    sol = _solver(params, scene)
    sol.step()
    assert sol.last_stats["iterations"] == max_loop + 1
    assert sol.last_stats["flags"] & _lib.SPH_F_NOT_CONVERGED
    x, v, p = sol.x.numpy(), sol.v.numpy(), sol.p.numpy()
    psi = sol.boundary_phi.numpy()
    dt = sol.dt
    sol.step()
    assert sol.last_stats["iterations"] == max_loop + 1
    ref = _oracle_step(oracle, params, x, v, scene.boundary_x, psi, dt, 1.0 / dt, p=p, warm_start=2,
                       fixed_iters=max_loop)
    assert_matches_oracle(oracle, sol, params, (x, v, scene.boundary_x, psi, dt), ref, ("p", "v", "x"),
                          p=p, warm_start=2)
    # without warm_continue the second step starts from the network's prediction
    plain = _solver(params.replace(warm_continue=False), scene)
    plain.steps(2)
    assert normrel(plain.p.numpy(), ref["p"]) > 100 * RTOL
    # a new state set after a capped solve starts from the prediction, as a
    # context without that history does
    x2, v2, dt2 = sol.x.numpy(), sol.v.numpy(), sol.dt
    assert sol.last_stats["flags"] & _lib.SPH_F_NOT_CONVERGED
    fresh = _solver(params, scene)
    for s_ in (sol, fresh):
        s_.set_state(x2, v2)
        s_.set_dt(dt2, 1.0 / dt2)
        s_.step()
    assert np.array_equal(sol.p.numpy(), fresh.p.numpy())
    assert np.array_equal(sol.x.numpy(), fresh.x.numpy())
    sol.close()
    plain.close()
    fresh.close()


def test_deterministic_and_graph_equivalent():
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    scene = preset_scene("dam_break_8k")
    outs = []
    for use_graph in (True, True, False):
        sol = _solver(preset_params("dam_break_8k", use_graph=use_graph), scene)
        sol.steps(10)
        outs.append((sol.x.numpy(), sol.v.numpy(), sol.p.numpy()))
        sol.close()
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)
    for a, b in zip(outs[0], outs[2]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("with_p", [True, False])
def test_host_round_trip_steps_on_exactly(with_p):
    """sph_get_fluid then sph_update_fluid (x, v and p, or x and v with the
    pressures kept on the device) between two steps changes nothing: the
    run goes on bit for bit as without the round trip (learned start with
    continuation after capped solves, so the pressure history matters)."""
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    scene = preset_scene("dam_break_8k")
    params = preset_params("dam_break_8k", warm_start="mlp", warm_continue=True)
    outs = []
    for trip in (False, True):
        sol = _solver(params, scene)
        sol.steps(3)
        for _ in range(5):
            if trip:
                x, v, p = sol.x.numpy(), sol.v.numpy(), sol.p.numpy()
                sol.update_state(x, v, p if with_p else None)
            sol.step()
        hist = [(h["iterations"], h["avg_err"], h["dt"]) for h in sol.stats_history(8)]
        outs.append((hist, sol.x.numpy(), sol.v.numpy(), sol.p.numpy()))
        sol.close()
    assert outs[0][0] == outs[1][0]
    for a, b in zip(outs[0][1:], outs[1][1:]):
        assert np.array_equal(a, b)


def test_texture_gathers_equal_plain_loads():
    """The solve's second pass (neighbour positions) and the neighbour
    build's second phase (positions, velocities) read through the texture
    path by default; the values are the same words, so every step is the
    same as with plain loads, bit for bit (learned start, continuation)."""
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    scene = preset_scene("dam_break_8k")
    outs = []
    for plain in (False, True):
        sol = _solver(preset_params("dam_break_8k", warm_start="mlp", warm_continue=True, plain_loads=plain),
                      scene)
        sol.steps(25)
        outs.append((sol.x.numpy(), sol.v.numpy(), sol.p.numpy(), sol.last_stats["iterations"]))
        sol.close()
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


def test_capacity_auto_grow():
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    scene = preset_scene("dam_break_8k")
    a = _solver(preset_params("dam_break_8k"), scene)
    b = _solver(preset_params("dam_break_8k", max_ff=4, max_fb=4, keep_fb_lists=True), scene)
    a.steps(3)
    b.steps(3)
    assert np.array_equal(a.x.numpy(), b.x.numpy())
    assert np.array_equal(a.p.numpy(), b.p.numpy())
    a.close()
    b.close()


def test_empty_fluid_and_isolated_particle(oracle):
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import Scene, box_boundary

    params = SolverParams(diameter=0.05)
    bx = box_boundary((0.5, 0.5, 0.5), 0.05, 2).astype(np.float32)
    empty = Scene(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), bx, len(bx), (0.5, 0.5, 0.5))
    sol = _solver(params, empty)
    sol.step()
    assert sol.last_stats["iterations"] == 2 and sol.last_stats["avg_err"] == 0.0
    sol.close()
    # one particle far from everything: a_ii = 0 takes the sign(0) * INV_SMALL branch
    x = np.array([[0.25, 0.3, 0.25]], np.float32)
    lone = Scene(x, np.zeros_like(x), bx, len(bx), (0.5, 0.5, 0.5))
    sol = _solver(params, lone)
    sol.step()
    psi = sol.boundary_phi.numpy()
    ref = _oracle_step(oracle, params, x, np.zeros_like(x), bx, psi, params.dt_max, 1 / params.dt_max)
    assert ref["p"][0] > 1e8
    assert sol.last_stats["iterations"] == ref["iterations"]
    assert_matches_oracle(oracle, sol, params, (x, np.zeros_like(x), bx, psi, params.dt_max), ref,
                          ("rho", "a_ii", "p", "v", "x"))
    sol.close()


def test_particles_outside_grid_domain(oracle):
    """Particles far outside the grid are clamped into edge cells; their
    neighbour sets must still be exact."""
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import dam_break

    params = SolverParams(diameter=0.02, w_table_size=1024, g_table_size=1024, keep_fb_lists=True,
                          domain_min=(0.0, 0.0, 0.0), domain_max=(0.2, 0.2, 0.2))
    sc = dam_break(fluid=(8, 8, 8), spacing=0.02, box=(0.4, 0.3, 0.3), jitter=1e-4, layers=2, seed=3)
    x = sc.fluid_x.copy()
    x[:64] += np.array([0.5, 0.0, 0.0], np.float32)   # beyond the grid's x extent
    x[64:80] -= np.array([0.0, 0.0, 0.3], np.float32)  # beyond the grid's low z side
    sc.fluid_x = x
    sol = _solver(params, sc)
    sol.neighbor_search()
    nb = sol.get_neighbors(with_boundary=True)
    op = oracle.reference_params(diameter=0.02, w_size=1024, g_size=1024)
    off, idx = oracle.neighbors(op, x, x, same=True)
    assert csr_equal(nb["ff_off"], nb["ff_idx"], off, idx)
    off, idx = oracle.neighbors(op, x, sc.boundary_x, same=False)
    assert csr_equal(nb["fb_off"], nb["fb_idx"], off, idx)
    sol.close()


def test_nonfinite_input_raises():
    from warpsph_b200._lib import SPH_E_NONFINITE, SphError
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    sc = preset_scene("dam_break_8k")
    sol = _solver(preset_params("dam_break_8k"), sc)
    v = sc.fluid_v.copy()
    v[123] = np.nan
    sol.set_state(sc.fluid_x, v)
    with pytest.raises(SphError) as e:
        sol.step()
    assert e.value.code == SPH_E_NONFINITE
    sol.close()


def test_no_boundary_free_fall_vs_oracle(oracle):
    """A fluid block with no boundary particles at all (nb = 0): the build
    skips the boundary grid and the solve has no boundary terms."""
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import Scene, dam_break

    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024)
    block = dam_break(fluid=(10, 10, 10), spacing=0.02, box=(0.4, 0.4, 0.4), jitter=1e-4, layers=2, seed=11)
    x = block.fluid_x.copy()
    sc = Scene(x, np.zeros_like(x), np.zeros((0, 3), np.float32), 0, (0.4, 0.4, 0.4))
    sol = _solver(params, sc)
    ref = _oracle_step(oracle, params, x, np.zeros_like(x), np.zeros((0, 3), np.float32),
                       np.zeros(0, np.float32), params.dt_max, 1 / params.dt_max)
    sol.step()
    nb = sol.get_neighbors()
    assert csr_equal(nb["ff_off"], nb["ff_idx"], ref["ff_off"], ref["ff_idx"])
    inputs = (x, np.zeros_like(x), np.zeros((0, 3), np.float32), np.zeros(0, np.float32), params.dt_max)
    assert_matches_oracle(oracle, sol, params, inputs, ref, ("rho", "rho_adv", "a_ii"))
    assert abs(sol.last_stats["iterations"] - ref["iterations"]) <= 1
    src = _at_reference_count(sol, params, sc, x, np.zeros_like(x), params.dt_max, ref)
    assert_matches_oracle(oracle, src, params, inputs, ref, ("p", "v", "x"))
    if src is not sol:
        src.close()
    sol.close()


def test_coincident_particles_vs_oracle(oracle):
    """Pairs of particles at exactly the same position: they are neighbours
    (r = 0 < h), contribute W(0) to each other's density and, with a zero
    direction, no gradient term (the reference's r < 1e-10 guard).  The
    reference itself turns such a pair into NaN: predict_v_adv divides by
    r^2 before multiplying the laplacian by VIS_MU = 0 (IISPH.py:273-278), and
    the oracle, which restates it expression for expression, does the same.
    The library drops that zero term (v_adv = v - g dt y exactly), so the
    step stays finite."""
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import Scene, box_boundary, dam_break

    params = SolverParams(diameter=0.02, gravity=9.81, w_table_size=1024, g_table_size=1024, fixed_iters=5)
    block = dam_break(fluid=(8, 8, 8), spacing=0.02, box=(0.3, 0.3, 0.3), jitter=1e-4, layers=2, seed=12)
    x = np.concatenate([block.fluid_x, block.fluid_x[::37]]).astype(np.float32)  # 14 exact duplicates
    bx = box_boundary((0.3, 0.3, 0.3), 0.02, 2).astype(np.float32)
    sc = Scene(x, np.zeros_like(x), bx, len(bx), (0.3, 0.3, 0.3))
    sol = _solver(params, sc)
    psi = sol.boundary_phi.numpy()
    ref = _oracle_step(oracle, params, x, np.zeros_like(x), bx, psi, params.dt_max, 1 / params.dt_max,
                       fixed_iters=5)
    sol.step()
    nb = sol.get_neighbors()
    assert csr_equal(nb["ff_off"], nb["ff_idx"], ref["ff_off"], ref["ff_idx"])
    assert_elem(sol.rho.numpy(), ref["rho"], parity_floors(params, params.dt_max)["rho"], "rho")  # no r^2 division
    dup = np.arange(0, len(block.fluid_x), 37)
    assert np.isnan(ref["v_adv"][dup]).all()             # the reference's 0 * inf
    v_adv = sol.v_adv.numpy()
    want = np.zeros_like(v_adv)
    want[:, 1] = np.float32(-params.gravity) * np.float32(params.dt_max)
    assert np.array_equal(v_adv, want)
    for f in ("p", "v", "x"):
        assert np.isfinite(getattr(sol, f).numpy()).all()
    assert sol.last_stats["iterations"] == 5
    sol.close()
