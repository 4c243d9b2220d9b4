"""Per-element parity of the CUDA path against the CPU oracle, per quantity.

Test infrastructure (imports the oracle).  For a fluid state it runs one
reference step (IISPH.py:1002-1371) three ways from identical inputs:

  * the FP32 oracle at its own iteration count (the reference's loop rule);
  * the FP64 oracle ("truth") with exactly that many Jacobi iterations;
  * the library through its C ABI; when its own convergence test stops one
    iteration away from the FP32 oracle's, a twin context with that many fixed
    iterations is stepped from the same inputs, so p, s, Ap, v and x are always
    compared at the reference's iteration count.

and reports per quantity the per-element relative error (tests.helpers.elemrel,
with the floors of tests.helpers.parity_floors): max and 99.9th percentile,
for GPU vs FP32 oracle, GPU vs FP64 oracle and FP32 oracle vs FP64 oracle.

    python -m tests.parity_table [--steps 200] [--out table.json]

runs the 8,000-particle dam break step by step for 200 steps (the demo loop of
scenes/IISPH_demo.py:57-66: every step from the state the previous one left)
and one step of the 1,000,000-particle dam break 30 steps in, and prints the
table (needs a CUDA GPU).
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from tests.helpers import csr_equal, elemstats, parity_floors  # noqa: E402

# quantity -> (library attribute, oracle key)
QUANTITIES = {
    "rho": ("rho", "rho"), "rho_adv": ("rho_adv", "rho_adv"), "v_adv": ("v_adv", "v_adv"),
    "d_ii": ("term_d_ii", "d_ii"), "a_ii": ("term_a_ii", "a_ii"), "s": ("sum_d_ij_p_j", "s"),
    "Ap": ("term_Ap_i", "Ap"), "p": ("p", "p"), "v": ("v", "v"), "x": ("x", "x"),
}
# computed before the Jacobi loop: independent of the iteration count
PRE_SOLVE = ("rho", "rho_adv", "v_adv", "d_ii", "a_ii")


def _oracle_params(oracle, params):
    return oracle.reference_params(diameter=params.diameter, gravity=params.gravity, w_size=params.w_table_size,
                                   g_size=params.g_table_size, vis_mu_scale=params.vis_mu_scale)


def oracle_pair(oracle, params, x, v, bx, psi, dt, fixed_iters=-1):
    """(FP32 oracle step, FP64 oracle step at the FP32 step's iteration count)."""
    from warpsph_b200.tables import kernel_tables

    op = _oracle_params(oracle, params)
    ref = oracle.step(op, x, v, bx, None, psi, dt, 1.0 / dt, tables=kernel_tables(params), fixed_iters=fixed_iters)
    truth = oracle.step(op, x, v, bx, None, psi, dt, 1.0 / dt, tables=oracle.kernel_tables(op, np.float64),
                        precision="f64", fixed_iters=int(ref["iterations"]))
    return ref, truth


def library_outputs(sol):
    return {q: np.asarray(getattr(sol, attr).numpy()) for q, (attr, _) in QUANTITIES.items()}


def compare(got, ref, truth, floors):
    """Per quantity: {"gpu_f32": (max, p999), "gpu_f64": ..., "f32_f64": ...}."""
    out = {}
    for q, (_, key) in QUANTITIES.items():
        fl = floors[q]
        xl = q == "x"
        r, t = ref[key], truth[key]
        out[q] = {"gpu_f32": elemstats(got[q], r, fl, xl), "gpu_f64": elemstats(got[q], t, fl, xl),
                  "f32_f64": elemstats(r, t, fl, xl)}
    return out


class StepChecker:
    """Steps a library solver from its own state and checks every step against
    the oracle from the same inputs (x, v, dt); a twin context with fixed
    iterations covers steps whose iteration count differs by one."""

    def __init__(self, oracle, params, scene):
        from warpsph_b200.solver import IISPH

        self.oracle = oracle
        self.params = params.replace(keep_fb_lists=True)
        self.scene = scene
        self.sol = IISPH(stage_path=None, params=self.params, scene=scene)
        self.psi = self.sol.boundary_phi.numpy()
        self.bx = scene.boundary_x
        self.twins = 0

    def advance(self, count):
        if count:
            self.sol.steps(count)

    def check_step(self):
        """One library step against the oracle.  Returns (record, comparison)."""
        from warpsph_b200.solver import IISPH

        sol = self.sol
        x, v, dt = sol.x.numpy(), sol.v.numpy(), sol.dt
        ref, truth = oracle_pair(self.oracle, self.params, x, v, self.bx, self.psi, dt)
        sol.step()
        nb = sol.get_neighbors(with_boundary=True)
        rec = {"iterations": int(sol.last_stats["iterations"]), "iterations_ref": int(ref["iterations"]),
               "ff_exact": bool(csr_equal(nb["ff_off"], nb["ff_idx"], ref["ff_off"], ref["ff_idx"])),
               "fb_exact": bool(csr_equal(nb["fb_off"], nb["fb_idx"], ref["fb_off"], ref["fb_idx"])),
               "dt_next": float(sol.dt), "dt_next_ref": float(ref["dt_next"]), "twin": False}
        got = library_outputs(sol)
        if rec["iterations"] != rec["iterations_ref"]:
            twin = IISPH(stage_path=None, params=self.params.replace(fixed_iters=rec["iterations_ref"]),
                         scene=self.scene)
            twin.set_state(x, v)
            twin.set_dt(dt, 1.0 / dt)
            twin.step()
            assert twin.last_stats["iterations"] == rec["iterations_ref"]
            twin_out = library_outputs(twin)
            for q in QUANTITIES:
                if q not in PRE_SOLVE:
                    got[q] = twin_out[q]
            twin.close()
            rec["twin"] = True
            self.twins += 1
        floors = parity_floors(self.params, dt)
        return rec, compare(got, ref, truth, floors)

    def close(self):
        self.sol.close()


def merge(acc, cmp):
    """Running maxima of (max, p999) per quantity and comparison."""
    for q, d in cmp.items():
        a = acc.setdefault(q, {})
        for k, (mx, p) in d.items():
            om, op_ = a.get(k, (0.0, 0.0))
            a[k] = (max(om, mx), max(op_, p))
    return acc


def run_dam_break_8k(oracle, steps=200):
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    chk = StepChecker(oracle, preset_params("dam_break_8k"), preset_scene("dam_break_8k"))
    acc, recs = {}, []
    for _ in range(steps):
        rec, cmp = chk.check_step()
        recs.append(rec)
        merge(acc, cmp)
    chk.close()
    return acc, recs, chk.twins


def run_dam_break_1m(oracle, warm=30):
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene

    chk = StepChecker(oracle, preset_params("dam_break_1m"), preset_scene("dam_break_1m"))
    chk.advance(warm)
    rec, cmp = chk.check_step()
    chk.close()
    return cmp, rec


def markdown(tables):
    lines = ["| quantity | floor | workload | GPU vs FP32 oracle: max / p99.9 | GPU vs FP64 oracle: max / p99.9 "
             "| FP32 oracle vs FP64 oracle: max / p99.9 |", "|---|---|---|---|---|---|"]
    for name, (acc, floors) in tables.items():
        for q in QUANTITIES:
            d = acc[q]
            cell = lambda k: f"{d[k][0]:.2e} / {d[k][1]:.2e}"  # noqa: E731
            lines.append(f"| {q} | {floors[q]:.3g} | {name} | {cell('gpu_f32')} | {cell('gpu_f64')} "
                         f"| {cell('f32_f64')} |")
    return "\n".join(lines)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--out", default=None)
    ap.add_argument("--skip-1m", action="store_true")
    a = ap.parse_args()
    from oracle import oracle
    from warpsph_b200.params import preset_params

    oracle.build()
    acc8, recs8, twins8 = run_dam_break_8k(oracle, a.steps)
    p8 = preset_params("dam_break_8k")
    tables = {f"dam break 8k, {a.steps} steps": (acc8, parity_floors(p8, p8.dt_max))}
    result = {"dam_break_8k": {"stats": acc8, "steps": recs8, "twins": twins8}}
    if not a.skip_1m:
        cmp1, rec1 = run_dam_break_1m(oracle)
        p1 = preset_params("dam_break_1m")
        tables["dam break 1M, step 30"] = (cmp1, parity_floors(p1, p1.dt_max))
        result["dam_break_1m"] = {"stats": cmp1, "step": rec1}
    print(markdown(tables))
    it = [(r["iterations"], r["iterations_ref"]) for r in recs8]
    print("8k: iteration differences", sorted({b - c for b, c in it}), "twins", twins8,
          "ff exact", all(r["ff_exact"] for r in recs8), "fb exact", all(r["fb_exact"] for r in recs8))
    if a.out:
        Path(a.out).write_text(json.dumps(result, indent=1))


if __name__ == "__main__":
    main()
