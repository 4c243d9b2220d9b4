"""Pin the CPU oracle to the reference: golden vectors produced by running the
reference's own kernel code (IISPH.py, sph_funcs.py) under an emulated Warp
runtime (tests/golden/make_golden.py).  No GPU needed."""
import numpy as np
import pytest

from tests.helpers import (csr_equal, elemstats, golden_oracle_params, golden_solver_params, jacobi_output_ok,
                           load_golden, normrel, parity_floors)

SCENES = ["ref_lattice", "dam_jitter", "compressed", "viscous"]


@pytest.mark.parametrize("name", SCENES)
def test_tables_bit_exact(oracle, name):
    G, meta = load_golden(name)
    P = golden_oracle_params(oracle, meta)
    w, g = oracle.kernel_tables(P)
    assert np.array_equal(w, G["W_table"])
    assert np.array_equal(g, G["grad_W_table"])


@pytest.mark.parametrize("name", SCENES)
def test_boundary_psi(oracle, name):
    G, meta = load_golden(name)
    P = golden_oracle_params(oracle, meta)
    psi = oracle.boundary_psi(P, G["boundary_x"], tables=(G["W_table"], G["grad_W_table"]))
    assert normrel(psi, G["boundary_phi"]) < 1e-6


@pytest.mark.parametrize("name", SCENES)
def test_steps_match_reference(oracle, name):
    G, meta = load_golden(name)
    P = golden_oracle_params(oracle, meta)
    tabs = (G["W_table"], G["grad_W_table"])
    for s in range(int(G["steps"])):
        pre = f"s{s}_"
        r = oracle.step(P, G[pre + "x_in"], G[pre + "v_in"], G["boundary_x"], None, G["boundary_phi"],
                        float(G[pre + "dt_in"]), float(G[pre + "inv_dt_in"]), tables=tabs, err_fp32_seq=True)
        assert csr_equal(r["ff_off"], r["ff_idx"], G[pre + "ff_off"], G[pre + "ff_idx"])
        assert csr_equal(r["fb_off"], r["fb_idx"], G[pre + "fb_off"], G[pre + "fb_idx"])
        assert r["iterations"] == int(G[pre + "iterations"])
        assert abs(r["avg_err"] - float(G[pre + "avg_err"])) < 1e-4 * float(G[pre + "avg_err"]) + 1e-12
        for key, gkey, tol in (("rho", "rho", 1e-6), ("rho_adv", "rho_adv", 1e-6), ("v_adv", "v_adv", 1e-6),
                               ("d_ii", "d_ii", 1e-5), ("a_ii", "a_ii", 1e-5), ("p", "p", 2e-5),
                               ("s", "s", 2e-5), ("Ap", "Ap", 2e-5), ("v", "v_out", 2e-5), ("x", "x_out", 1e-6)):
            assert normrel(r[key], G[pre + gkey]) < tol, (name, s, key, normrel(r[key], G[pre + gkey]))
        assert r["dt_next"] == float(G[pre + "dt_out"])
        # per element: pre-solve terms to float32 summation order, the
        # Jacobi outputs to the FP32 noise floor (tests.helpers.jacobi_output_ok)
        fl = parity_floors(golden_solver_params(meta), float(G[pre + "dt_in"]))
        for key in ("rho", "rho_adv", "v_adv", "d_ii", "a_ii"):
            assert elemstats(r[key], G[pre + key], fl[key])[0] < 5e-6, (name, s, key)
        assert elemstats(r["v"], G[pre + "v_out"], fl["v"])[0] < 1e-4, (name, s)
        assert elemstats(r["x"], G[pre + "x_out"], fl["x"], x_like=True)[0] < 1e-4, (name, s)
        if s == 0:
            t = oracle.step(P, G[pre + "x_in"], G[pre + "v_in"], G["boundary_x"], None, G["boundary_phi"],
                            float(G[pre + "dt_in"]), float(G[pre + "inv_dt_in"]),
                            tables=oracle.kernel_tables(P, np.float64), precision="f64",
                            fixed_iters=int(G[pre + "iterations"]))
            for key in ("p", "s", "Ap"):
                ok, detail = jacobi_output_ok(r[key], G[pre + key], t[key], fl[key])
                assert ok, (name, key, detail)


def test_fp64_truth_close_to_fp32(oracle):
    """The FP32 mirror and the FP64 truth agree to float32 accuracy on a golden state."""
    G, meta = load_golden("dam_jitter")
    P = golden_oracle_params(oracle, meta)
    args = (G["s0_x_in"], G["s0_v_in"], G["boundary_x"], None, G["boundary_phi"], float(G["s0_dt_in"]))
    r32 = oracle.step(P, *args, fixed_iters=8)
    r64 = oracle.step(P, *args, precision="f64", fixed_iters=8)
    assert normrel(r32["rho"], r64["rho"]) < 1e-6
    assert normrel(r32["p"], r64["p"]) < 1e-4
    assert normrel(r32["x"], r64["x"]) < 1e-6
