"""Generate golden IISPH step vectors by running the reference's own solver.

Test infrastructure only.  The reference (Mo-ZheHan/WarpSPH, read from a local
checkout given by ``--reference``) is pure Python on NVIDIA Warp, which is
not installed here.  This script imports the reference's own modules
(``wp_sph/main.py``, ``wp_sph/solver/sph_funcs.py``, ``wp_sph/solver/IISPH.py``)
with ``warp`` replaced by the numpy emulation in ``warp_emu.py``, patches the
module-level scene constants the reference reads at import time
(``wp_sph/main.py:25-61``, ``sph_funcs.py:43-44``), optionally injects a
jittered state, and records per-step inputs and outputs of ``IISPH.step()``
(``IISPH.py:1002-1371``) into ``tests/golden/<scene>.npz``.

Usage:  python tests/golden/make_golden.py --reference PATH [scene ...]
"""

from __future__ import annotations

import argparse
import importlib
import json
import math
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import warp_emu  # noqa: E402

# Scenes: constants patched into wp_sph/main.py before the solver is imported.
SCENES = {
    # The reference's own EMPTY scene recipe (IISPH.py:763-766, unjittered lattice,
    # 3 boundary layers, 8192/65536-sample tables) on a 0.5 m box.
    "ref_lattice": dict(diameter=0.05, box=(0.5, 0.5, 0.5), gravity=9.8,
                        w_size=8192, g_size=65536, steps=3, jitter=0.0, v0=(0.0, 0.0, 0.0),
                        isolated=False, compress=1.0, seed=0),
    # Dam-break style block: 0.02 m spacing, +-1e-4 m seeded jitter, 1024-sample
    # tables, g = 9.81, an initial downward velocity and one isolated particle
    # (a_ii = 0, exercising IISPH.py:535-536).
    "dam_jitter": dict(diameter=0.02, box=(0.4, 0.24, 0.16), gravity=9.81,
                       w_size=1024, g_size=1024, steps=4, jitter=1e-4, v0=(0.0, -0.5, 0.0),
                       isolated=True, compress=1.0, seed=1),
    # Lattice compressed to 0.9 of its spacing toward the floor: the pressure
    # solve runs many Jacobi iterations from the first step.
    "compressed": dict(diameter=0.05, box=(0.5, 0.5, 0.5), gravity=9.8,
                       w_size=8192, g_size=65536, steps=3, jitter=2e-4, v0=(0.0, 0.0, 0.0),
                       isolated=False, compress=0.9, seed=2),
    # The dam-break block with viscosity on (VIS_MU = 0.01 RHO_0, main.py:61):
    # the laplacian of predict_v_adv (IISPH.py:248-278) acts on the jittered
    # velocities from the first step.
    "viscous": dict(diameter=0.02, box=(0.4, 0.24, 0.16), gravity=9.81,
                    w_size=1024, g_size=1024, steps=3, jitter=1e-4, v0=(0.2, -0.5, 0.1),
                    isolated=False, compress=1.0, seed=4, vis_mu_scale=0.01),
}


def _stub_modules():
    """trimesh and joblib are only used by mesh scenes (model.py); stub them."""
    tm = types.ModuleType("trimesh")
    tm.Trimesh = object
    sys.modules["trimesh"] = tm
    jl = types.ModuleType("joblib")

    class Memory:
        def __init__(self, *a, **k):
            pass

        def cache(self, f):
            return f

    jl.Memory = Memory
    jl.Parallel = None
    jl.delayed = None
    sys.modules["joblib"] = jl


def load_reference(ref: Path, cfg: dict):
    for name in [m for m in sys.modules if m.startswith("wp_sph_ref")]:
        del sys.modules[name]
    warp_emu.install()
    _stub_modules()
    pkg = types.ModuleType("wp_sph_ref")
    pkg.__path__ = [str(ref / "wp_sph")]
    sys.modules["wp_sph_ref"] = pkg
    main = importlib.import_module("wp_sph_ref.main")
    # scene constants (main.py:25-53) and the derived ones (main.py:57-61)
    d = cfg["diameter"]
    main.DIAMETER = d
    main.GRAVITY = cfg["gravity"]
    main.BOX_WIDTH, main.BOX_HEIGHT, main.BOX_LENGTH = cfg["box"]
    main.SMOOTHING_LENGTH = 2 * d
    main.TIME_STEP_MAX = 5e-2 * d
    main.FLUID_MASS = main.RHO_0 * d**3
    main.SIGMA = 8 / (math.pi * main.SMOOTHING_LENGTH**3)
    main.VIS_MU = cfg.get("vis_mu_scale", 0.0) * main.RHO_0
    spkg = types.ModuleType("wp_sph_ref.solver")
    spkg.__path__ = [str(ref / "wp_sph" / "solver")]
    sys.modules["wp_sph_ref.solver"] = spkg
    funcs = importlib.import_module("wp_sph_ref.solver.sph_funcs")
    funcs.W_SIZE = cfg["w_size"]
    funcs.GRAD_W_SIZE = cfg["g_size"]
    funcs.precompute_tables()
    solver = importlib.import_module("wp_sph_ref.solver.IISPH")
    return main, funcs, solver


def _sets(num, index, lst, n):
    off = np.zeros(n + 1, dtype=np.int64)
    idx = []
    for i in range(n):
        seg = np.sort(lst[index[i]: index[i] + num[i]])
        idx.append(seg)
        off[i + 1] = off[i] + len(seg)
    return off, (np.concatenate(idx) if idx else np.zeros(0)).astype(np.int32)


def run_scene(ref: Path, name: str, cfg: dict) -> dict:
    main, funcs, mod = load_reference(ref, cfg)
    counts = {"update_p": 0}
    real_launch = warp_emu.launch

    def counting_launch(kernel, dim, inputs=(), outputs=(), device=None):
        counts[kernel.__name__] = counts.get(kernel.__name__, 0) + 1
        return real_launch(kernel, dim, inputs, outputs, device)

    mod.wp.launch = counting_launch
    sph = mod.IISPH(stage_path=None, preview=False, verbose=False)

    rng = np.random.default_rng(cfg["seed"])
    x = sph.x.numpy().astype(np.float64)
    if cfg["compress"] != 1.0:
        x = x * cfg["compress"]
    if cfg["jitter"] > 0:
        x = x + rng.uniform(-cfg["jitter"], cfg["jitter"], size=x.shape)
    if cfg["isolated"]:
        x[-1] = (cfg["box"][0] * 0.5, cfg["box"][1] * 0.85, cfg["box"][2] * 0.5)
    sph.x.assign(x.astype(np.float32))
    v = np.zeros_like(x) + np.array(cfg["v0"])
    if cfg["jitter"] > 0:
        v = v + rng.uniform(-0.05, 0.05, size=v.shape)
    sph.v.assign(v.astype(np.float32))

    out = {
        "meta": json.dumps({
            "scene": name, **{k: v for k, v in cfg.items() if k != "box"}, "box": list(cfg["box"]),
            "rho0": main.RHO_0, "omega": main.OMEGA, "eta": main.ETA, "inv_small": main.INV_SMALL,
            "h": main.SMOOTHING_LENGTH, "dt_max": main.TIME_STEP_MAX, "fluid_mass": main.FLUID_MASS,
            "sigma": main.SIGMA, "vis_mu": main.VIS_MU, "n": sph.n, "boundary_n": sph.boundary_n,
            "generator": "tests/golden/make_golden.py (reference kernels under warp_emu)",
        }),
        "boundary_x": sph.boundary_x.numpy(),
        "boundary_phi": sph.boundary_phi.numpy(),
        "W_table": funcs.W_table.numpy(),
        "grad_W_table": funcs.grad_W_table.numpy(),
    }
    for s in range(cfg["steps"]):
        pre = f"s{s}_"
        out[pre + "x_in"] = sph.x.numpy()
        out[pre + "v_in"] = sph.v.numpy()
        out[pre + "dt_in"] = np.float64(sph.dt)
        out[pre + "inv_dt_in"] = np.float64(sph.inv_dt)
        counts["update_p"] = 0
        sph.step()
        n = sph.n
        out[pre + "ff_off"], out[pre + "ff_idx"] = _sets(
            sph.ff_neighbor_num.numpy(), sph.ff_neighbor_list_index.numpy(), sph.ff_neighbor_list.numpy(), n)
        out[pre + "fb_off"], out[pre + "fb_idx"] = _sets(
            sph.fs_neighbor_num.numpy(), sph.fs_neighbor_list_index.numpy(), sph.fs_neighbor_list.numpy(), n)
        out[pre + "rho"] = sph.rho.numpy()
        out[pre + "v_adv"] = sph.v_adv.numpy()
        out[pre + "rho_adv"] = sph.rho_adv.numpy()
        out[pre + "d_ii"] = sph.term_d_ii.numpy()
        out[pre + "a_ii"] = sph.term_a_ii.numpy()
        out[pre + "p"] = sph.p.numpy()
        out[pre + "s"] = sph.sum_d_ij_p_j.numpy()
        out[pre + "Ap"] = sph.term_Ap_i.numpy()
        out[pre + "iterations"] = np.int32(counts["update_p"])
        out[pre + "avg_err"] = np.float64(sph.average_rho_error)
        out[pre + "v_out"] = sph.v.numpy()
        out[pre + "x_out"] = sph.x.numpy()
        out[pre + "dt_out"] = np.float64(sph.dt)
        print(f"{name} step {s}: iters={counts['update_p']} avg_err={float(sph.average_rho_error):.3e} "
              f"p_max={float(out[pre + 'p'].max()):.4g}", flush=True)
    out["steps"] = np.int32(cfg["steps"])
    return out


def main_cli():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of a WarpSPH checkout")
    ap.add_argument("scenes", nargs="*", default=list(SCENES))
    args = ap.parse_args()
    ref = Path(args.reference)
    for name in args.scenes:
        data = run_scene(ref, name, SCENES[name])
        np.savez_compressed(HERE / f"{name}.npz", **data)
        print("wrote", HERE / f"{name}.npz")


if __name__ == "__main__":
    main_cli()
