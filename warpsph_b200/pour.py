"""Fluid poured onto a procedural obstacle (the uneven-occupancy workload).

    python -m warpsph_b200.pour [--max-particles N] [--steps-after K]

A 0.3 x 0.3 m inlet 1.8 m up in a 2 m cube emits layers of particles at
0.008 m spacing moving down at 2 m/s (one layer every 4 ms) onto the seeded
union of 6 boxes and 4 tori (scenes.pour_scene), until N fluid particles have
entered; then K more steps run with the emitter off.  The emitter appends each
layer on the device (IISPH.add_fluid), between batches of steps that end when
the next layer is due.  The reference has no emitter: its particle set is
fixed at init_particles (IISPH.py:857-1000).

The solve starts from the reference's p = 0 by default: the learned warm
start was trained on dam breaks, and on the 2M pour's late impacts it let
splash particles reach 105 m/s (p = 0: 15.6 m/s), stretching the CFL step.
"""

from __future__ import annotations

import argparse
import json
import time

from .params import POUR, pour_params
from .scenes import pour_scene
from .solver import IISPH


def emit_until(sol: IISPH, inlet, progress=None) -> int:
    """Step `sol` and feed it the inlet's layers until the inlet is done.
    Returns the number of steps taken."""
    taken = 0
    while not inlet.done:
        # steps until the next layer leaves the opening, at the current dt
        wait = inlet.layers * inlet.period - sol.sim_time
        k = max(1, int(wait / sol.dt + 0.999))
        sol.steps(k)
        taken += k
        x, v = inlet.due(sol.sim_time)
        sol.add_fluid(x, v)
        if progress:
            progress(sol, taken)
    return taken


def make(max_particles: int = POUR["max_particles"], seed: int = POUR["seed"], **param_kw):
    scene, inlet = pour_scene(seed=seed, spacing=POUR["diameter"], domain=POUR["domain"], layers=POUR["layers"])
    inlet.max_particles = max_particles
    sol = IISPH(stage_path=None, params=pour_params(**param_kw), scene=scene)
    return sol, inlet


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--max-particles", type=int, default=POUR["max_particles"])
    ap.add_argument("--steps-after", type=int, default=0)
    ap.add_argument("--warm", choices=["zero", "half", "mlp"], default="zero")
    a = ap.parse_args()
    sol, inlet = make(a.max_particles, warm_start=a.warm)
    t0 = time.perf_counter()
    steps = emit_until(sol, inlet)
    if a.steps_after:
        sol.steps(a.steps_after)
    print(json.dumps({"fluid": sol.n, "boundary": sol.boundary_n, "emission_steps": steps,
                      "steps_after": a.steps_after, "sim_time": sol.sim_time, "wall_s": time.perf_counter() - t0,
                      "last": sol.last_stats}))
    sol.close()


if __name__ == "__main__":
    main()
