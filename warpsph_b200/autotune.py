"""Autotuner for the kernel launch shapes.

Knobs: threads per block of the neighbour build (`block_size`), and of the
persistent pressure solve (`jacobi_block`), particles per solve thread
(`jacobi_ppt`, so one solve chunk holds jacobi_block * jacobi_ppt particles),
the unroll of the solve's neighbour loops (`jacobi_unroll`), and whether the
read-only neighbour gathers use the texture path or plain loads
(`plain_loads`).  None of them changes the arithmetic, only how work maps
onto the SMs and which load path carries it.

Each candidate runs the caller's own scene (or batch of scenes) on a fresh
solver: `warm` untimed steps, then `steps` steps timed with CUDA events.  The
build knob is tuned first with the solve at its default, then the solve knobs
jointly, then the load path at the best shape.  Results are cached in JSON
keyed by GPU name and workload size.
"""

from __future__ import annotations

import json
import os
from pathlib import Path

BUILD_BLOCKS = (64, 128, 256)
SOLVE_SHAPES = [(b, p, u) for b in (128, 256) for p in (1, 2) for u in (2, 4, 8)] + [(512, 1, 4), (1024, 1, 4)]
DEFAULT_SOLVE = (1024, 1, 4)  # the library's shape when SphParams leaves it 0
CACHE = Path(os.environ.get("WPSPH_AUTOTUNE_CACHE", Path.home() / ".cache" / "warpsph_b200" / "autotune.json"))


def _signature(scenes, params) -> str:
    n = sum(s.n for s in scenes)
    nb = sum(s.boundary_n for s in scenes)
    return f"scenes={len(scenes)},n={n},nb={nb},d={params.diameter},warm={params.warm_start},v3"


def _time(scenes, params, warm, steps) -> float:
    import torch

    from .batch import BatchIISPH

    b = BatchIISPH(scenes, params)
    b.prepare()
    if warm:
        b.steps(warm)
    st = torch.cuda.ExternalStream(b._lib.sph_stream(b._ctx))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    rc = b._lib.sph_launch_steps(b._ctx, steps)
    e1.record(st)
    e1.synchronize()
    b.close()
    if rc != 0:
        raise RuntimeError(f"sph_launch_steps failed ({rc})")
    return e0.elapsed_time(e1) / steps


def autotune(scenes, params, warm=10, steps=20, use_cache=True, verbose=False) -> dict:
    """Best knob values for this workload: {'block_size', 'jacobi_block',
    'jacobi_ppt', 'jacobi_unroll', 'plain_loads', 'ms_per_step', 'trials'}."""
    import torch

    key = f"{torch.cuda.get_device_name(params.device)}|{_signature(scenes, params)}"
    cache = {}
    if use_cache and CACHE.exists():
        cache = json.loads(CACHE.read_text())
        if key in cache:
            return cache[key]
    trials = []
    best_build, best_t = 128, float("inf")
    for bb in BUILD_BLOCKS:
        t = _time(scenes, params.replace(block_size=bb), warm, steps)
        trials.append({"block_size": bb, "ms": t})
        if verbose:
            print("build", bb, t)
        if t < best_t:
            best_build, best_t = bb, t
    # the build sweep ran the solve at the caller's shape (the library's
    # default where unset), so best_t is that shape's time: a solve shape must
    # beat it to replace it
    best = (params.jacobi_block or DEFAULT_SOLVE[0], params.jacobi_ppt or DEFAULT_SOLVE[1],
            params.jacobi_unroll or DEFAULT_SOLVE[2])
    for blk, ppt, unr in SOLVE_SHAPES:
        t = _time(scenes, params.replace(block_size=best_build, jacobi_block=blk, jacobi_ppt=ppt,
                                         jacobi_unroll=unr), warm, steps)
        trials.append({"jacobi_block": blk, "jacobi_ppt": ppt, "jacobi_unroll": unr, "ms": t})
        if verbose:
            print("solve", blk, ppt, unr, t)
        if t < best_t:
            best, best_t = (blk, ppt, unr), t
    shape = dict(block_size=best_build, jacobi_block=best[0], jacobi_ppt=best[1], jacobi_unroll=best[2])
    plain = bool(params.plain_loads)
    t = _time(scenes, params.replace(plain_loads=not plain, **shape), warm, steps)
    trials.append({"plain_loads": not plain, "ms": t})
    if verbose:
        print("plain_loads", not plain, t)
    if t < best_t:
        plain, best_t = not plain, t
    res = dict(shape, plain_loads=plain, ms_per_step=best_t, trials=trials)
    if use_cache:
        CACHE.parent.mkdir(parents=True, exist_ok=True)
        cache[key] = res
        CACHE.write_text(json.dumps(cache, indent=1))
    return res


def apply(params, tuned: dict):
    return params.replace(block_size=tuned["block_size"], jacobi_block=tuned["jacobi_block"],
                          jacobi_ppt=tuned["jacobi_ppt"], jacobi_unroll=tuned["jacobi_unroll"],
                          plain_loads=bool(tuned.get("plain_loads", params.plain_loads)))
