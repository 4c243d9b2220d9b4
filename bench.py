#!/usr/bin/env python
"""IISPH time-step benchmark on the 1,000,000-particle dam break (one B200).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one IISPH.step() (IISPH.py:1002-1371): cell sort, neighbour build
and advection prediction, the relaxed-Jacobi solve to 0.1 % average density
error, kick/drift and CFL.  The workload is the dam break of 100^3 fluid
particles at 0.01 m spacing with +-5e-5 m seeded jitter in a 2 x 1 x 1 m box
with 2 boundary layers (206,464 boundary particles), 1024-sample kernel tables,
g = 9.81, dt = 5e-4 s.  Inputs are synthetic (seeded); the state and neighbour
lists (~0.5 GB) exceed the 126 MB L2, so no flush is needed between steps.

Prints one JSON line (rank 0).  With torchrun (N > 1) every rank runs an
independent replica of the scene: the single-scene step does not shard
(replicas only), so there is no data-path collective; timing is the max over
ranks and `value` counts the steps of all ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "IISPH steps/s at 1M particles, 0.1% density err; learned warm-start vs plain"
PRESET = "dam_break_1m"
# cell_keys, scan_onepass, scatter, cell_sort, gather, build, jacobi
# (+ column_top and mlp_infer with the learned warm start)
KERNELS_PER_STEP = 7


def kernels_per_step(warm: str) -> int:
    return KERNELS_PER_STEP + (2 if warm.startswith("mlp") else 0)


def warm_kwargs(mode: str) -> dict:
    """SolverParams of a warm-start mode; "mlp_continue" is the learned start
    that, after a solve stopped at the iteration cap, continues from it."""
    if mode == "mlp_continue":
        return dict(warm_start="mlp", warm_continue=True)
    return dict(warm_start=mode)


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_config(K: int, world: int) -> dict:
    """The workload both arms run (same dict in both JSON lines)."""
    return {"workload": f"dam break, 1,000,000 fluid + 206,464 boundary particles, steps [0, {K}) "
                        "from the initial state, 0.1% avg density err",
            "preset": PRESET, "parallelism": f"replicas{world}",
            "l2": "working set > 126 MB L2 (no flush needed)"}


def settled_steps(iters, cap):
    """Timed steps after the last solve stopped by the iteration cap (the
    dam break's start-up transient)."""
    last_cap = max((k for k, it in enumerate(iters) if it >= cap), default=-1)
    return len(iters) - 1 - last_cap


def keep_timing(times, iters, K, budget_s, cap):
    """Whether the sampled CPU run times another step: until K are done or
    the budget is spent, and past the budget (up to 3x) until 5 steps after
    the transient are in, so untimed steps are never charged from capped
    solves."""
    t_total = sum(times)
    return len(times) < K and (not times or t_total < budget_s
                               or (settled_steps(iters, cap) < 5 and t_total < 3 * budget_s))


def sampled_value(times, iters, K, cap):
    """steps/s over K steps from the timed ones: untimed steps are charged at
    the median of the last (at most 20) timed steps after the transient (the
    median: the first of them may still be a long solve); with none, at the
    cheapest timed step.  Returns (value, the times the charge came from)."""
    timed, after = len(times), settled_steps(iters, cap)
    tail = list(times[timed - min(20, after):]) if after > 0 else [min(times)]
    t_rest = (K - timed) * float(np.median(tail)) if timed < K else 0.0
    return K / (sum(times) + t_rest), tail


def run_cpu_reference(budget_s: float, max_steps: int, nthreads: int = 0):
    """The reference algorithm (the CPU oracle: FP32, p <- 0 start, OpenMP on
    all host threads) on the same scene, steps [0, K) from the initial state.

    The steps are timed one by one as they run, until K are done or the time
    budget is spent.  value = K / (timed seconds) when all K ran; otherwise
    the remaining steps are charged at the median time of the last (at most
    20) timed steps after the start-up transient's capped solves, timing on
    past the budget (up to 3x) until 5 such steps are in, and the line says
    how many were timed.  That charge is a lower bound on the CPU's time, so
    the value errs on the CPU's side: those steps of the 1M dam break take 2
    iterations, while the p <- 0 solve averages about 7 per step over steps
    [45, 500) (3784 iterations over [0, 500) on the device, 681 of them in
    the first 45 steps).  Iteration counts
    are the oracle's own.  Two unit costs are reported beside it (a step with
    2 and one with 12 fixed iterations at the initial state), and the same
    2-iteration step on one thread."""
    from oracle import oracle
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.tables import kernel_tables

    oracle.build()
    params = preset_params(PRESET)
    scene = preset_scene(PRESET)
    op = oracle.reference_params(diameter=params.diameter, gravity=params.gravity, w_size=1024, g_size=1024)
    tabs = kernel_tables(params)
    nt = nthreads or oracle.max_threads()
    psi = oracle.boundary_psi(op, scene.boundary_x, tables=tabs, nthreads=nt)
    x0, v0, dt0 = scene.fluid_x.copy(), scene.fluid_v.copy(), params.dt_max

    def one(x, v, dt, fixed=-1, threads=None):
        t0 = time.perf_counter()
        r = oracle.step(op, x, v, scene.boundary_x, None, psi, dt, 1.0 / dt, tables=tabs, export=False,
                        nthreads=threads or nt, fixed_iters=fixed)
        return time.perf_counter() - t0, r

    K = max(1, max_steps)
    x, v, dt = x0, v0, dt0
    times, iters = [], []
    cap = 101  # iterations of a solve stopped by the reference's cap (loop > 100)
    while keep_timing(times, iters, K, budget_s, cap):
        t, r = one(x, v, dt)
        times.append(t)
        x, v, dt = r["x"], r["v"], r["dt_next"]
        iters.append(int(r["iterations"]))
    timed, t_total = len(times), sum(times)
    value, tail = sampled_value(times, iters, K, cap)

    t2, _ = one(x0, v0, dt0, fixed=2)
    t12, _ = one(x0, v0, dt0, fixed=12)
    t_iter = max((t12 - t2) / 10.0, 1e-9)
    t_base = max(t2 - 2.0 * t_iter, 0.0)
    t2_one, _ = one(x0, v0, dt0, fixed=2, threads=1)
    if timed == K:
        sample = (f"FP32 oracle (p <- 0, the reference algorithm), {nt} OpenMP threads, 1M-particle dam break: "
                  f"steps [0, {K}) from the initial state all timed ({sum(iters)} Jacobi iterations)")
    else:
        sample = (f"FP32 oracle (p <- 0, the reference algorithm), {nt} OpenMP threads, 1M-particle dam break: "
                  f"steps [0, {timed}) timed ({sum(iters)} Jacobi iterations), the other {K - timed} charged "
                  f"at the median of the last {len(tail)} timed steps after the capped start-up solves "
                  f"({np.median(tail) * 1e3:.0f} ms)")
    return {"value": value, "unit": "steps/s", "cores": nt, "kind": "port", "sample": sample,
            "timed_steps": timed, "timed_s": t_total, "iterations": iters,
            "unit_costs": {"ms_per_iteration": t_iter * 1e3, "ms_step_base": t_base * 1e3,
                           "model_steps_per_s": K / (K * t_base + sum(iters) / timed * K * t_iter)},
            "one_thread": {"ms_step_2_iterations": t2_one * 1e3, "threads_speedup": t2_one / t2}}


def bench_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    base = run_cpu_reference(budget_s=120.0, max_steps=max(1, args.steps))
    line = {
        "impl": "reference", "metric": METRIC, "value": base["value"], "unit": "steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / base["value"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.steps, args.gpus),
        "algorithm": "reference: pressure solve from p = 0 every step (IISPH.py:166-174)",
        "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_ours(args):
    import ctypes

    import torch

    from warpsph_b200 import _lib
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.solver import IISPH

    from warpsph_b200 import ranks

    rank, world, local = ranks.env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # N ranks = N independent replicas of the scene; only the timing is reduced
    dist = ranks.init("nccl", device=dev)

    scene = preset_scene(PRESET)
    n = scene.n
    headline = args.warm
    K = args.steps

    def fresh(mode):
        s = IISPH(stage_path=None, params=preset_params(PRESET, device=local, **warm_kwargs(mode)), scene=scene)
        _lib.check(s._ctx, s._lib.sph_prepare(s._ctx))  # capture the step graph outside any timing
        return s

    def stream_of(s):
        return torch.cuda.ExternalStream(s._lib.sph_stream(s._ctx), device=dev)

    # a dam break under gravity cannot outrun free fall from the box height:
    # a step faster than 10x that is a diverged run, not a measurement
    v_limit = 10.0 * (2.0 * 9.81 * scene.box[1]) ** 0.5

    def check_flags(hist, headline_run=True):
        flags = 0
        for h in hist:
            flags |= h["flags"]
        bad = _lib.SPH_F_TIMEOUT | _lib.SPH_F_NONFINITE | _lib.SPH_F_FF_OVERFLOW | _lib.SPH_F_FB_OVERFLOW
        if flags & bad:
            raise RuntimeError(f"step flags {flags:#x} in a timed region")
        vmax = max(h["v_max"] for h in hist)
        if headline_run and vmax > v_limit:
            raise RuntimeError(f"v_max {vmax:.3g} m/s exceeds {v_limit:.3g} m/s: the run diverged")

    def timed_steps(s, count, headline_run=True):
        st = stream_of(s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        _lib.check(s._ctx, s._lib.sph_launch_steps(s._ctx, count))
        e1.record(st)
        e1.synchronize()
        hist = s.stats_history(count)
        check_flags(hist, headline_run)
        return e0.elapsed_time(e1), hist

    # warm-up: W steps on a throwaway solver (clocks, module load, graph capture)
    w = fresh(headline)
    if args.warmup:
        w.steps(args.warmup)
    w.close()

    if args.profile:
        # minimal launch sequence for ncu: K steps from the initial state
        s = fresh(headline)
        _lib.check(s._ctx, s._lib.sph_launch_steps(s._ctx, K))
        torch.cuda.synchronize()
        hist = s.stats_history(K)
        print(json.dumps({"profile_run": True, "steps": K, "n": n,
                          "iterations": [h["iterations"] for h in hist],
                          "n_ff_pairs": [h["n_ff_pairs"] for h in hist]}))
        s.close()
        return

    # timed region: steps [0, K) of the dam break from its initial state
    sol = fresh(headline)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ms, hist = timed_steps(sol, K)
    clock = clocks.stop()
    sol.close()
    ms_max = ranks.max_over_ranks(ms, dist, dev)
    value = world * K / (ms_max / 1000.0)
    iters = [h["iterations"] for h in hist]

    # the same K steps with the other warm-start modes (context for the headline),
    # with the distribution over steps of the average density error at exit
    def mode_line(t_ms, hs):
        errs = np.array([h["avg_err"] for h in hs])
        return {"steps_per_s": K / (t_ms / 1000.0), "jacobi_iterations": int(sum(h["iterations"] for h in hs)),
                "v_max_max": float(max(h["v_max"] for h in hs)),
                "avg_density_err": {"p50": float(np.percentile(errs, 50)), "p90": float(np.percentile(errs, 90)),
                                    "p99": float(np.percentile(errs, 99)), "max": float(errs.max()),
                                    "steps_above_tol": int((errs > 1e-3).sum())}}

    modes = {}
    for mode in ("zero", "half", "mlp", "mlp_continue"):
        if mode == headline:
            modes[mode] = mode_line(ms, hist)
            continue
        s = fresh(mode)
        m_ms, m_hist = timed_steps(s, K, headline_run=False)
        s.close()
        modes[mode] = mode_line(m_ms, m_hist)

    # dominant kernel: per-launch CUDA-event time of the persistent solve over the same K steps
    s = fresh(headline)
    st = stream_of(s)
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(K)]
    torch.cuda.synchronize()
    for e in ev:
        e[0].record(st)
        _lib.check(s._ctx, s._lib.sph_launch_phase(s._ctx, 0))  # sort + neighbour build
        e[1].record(st)
        _lib.check(s._ctx, s._lib.sph_launch_phase(s._ctx, 2))  # warm-start inference
        e[2].record(st)
        e[3].record(st)
        _lib.check(s._ctx, s._lib.sph_launch_phase(s._ctx, 3))  # k_jacobi alone
        e[4].record(st)
    torch.cuda.synchronize()
    hk = s.stats_history(K)
    check_flags(hk)
    s.close()
    t_front = [e[0].elapsed_time(e[1]) for e in ev]
    t_warm = [e[1].elapsed_time(e[2]) for e in ev]
    t_jac = [e[3].elapsed_time(e[4]) for e in ev]
    bytes_launch = [h["iterations"] * (100.0 * n + 8.0 * h["n_ff_pairs"]) + 112.0 * n for h in hk]
    achieved = sum(bytes_launch) / (sum(t_jac) / 1000.0) / 1e9
    peak, peak_kind = _peaks()
    # DRAM traffic per launch: the ncu-measured ratio of dram bytes to these
    # algorithmic bytes on a captured k_jacobi launch, applied to this run's
    # mean launch (traffic grows with iterations x pairs like the bytes rule)
    traffic = None
    tf = ROOT / "profiles" / "jacobi_traffic.json"
    if tf.exists():
        ratio = json.loads(tf.read_text()).get("traffic_over_algorithmic")
        if ratio:
            traffic = ratio * sum(bytes_launch) / len(bytes_launch)

    # end to end through the C ABI with host buffers: every step uploads its
    # input state (x, v: the reference's state) from pinned memory with
    # sph_update_fluid (which, unlike sph_set_fluid, keeps the solver's
    # history, the pressures included: the headline's continuation after
    # capped solves runs as on the device), steps, and reads back x and v;
    # every step's flags and v_max are checked
    s = fresh(headline)
    L, ctx = s._lib, s._ctx
    hx = torch.from_numpy(scene.fluid_x.copy()).pin_memory()
    hv = torch.from_numpy(scene.fluid_v.copy()).pin_memory()
    stt = _lib.SphStepStats()
    vp = ctypes.c_void_p
    e2e_hist = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        _lib.check(ctx, L.sph_update_fluid(ctx, vp(hx.data_ptr()), vp(hv.data_ptr()), None, n))
        _lib.check(ctx, L.sph_step(ctx, ctypes.byref(stt)))
        _lib.check(ctx, L.sph_get_fluid(ctx, vp(hx.data_ptr()), vp(hv.data_ptr()), None, None, None))
        e2e_hist.append(stt.as_dict())
    e2e_s = time.perf_counter() - t0
    s.close()
    check_flags(e2e_hist)
    e2e_iters = int(sum(h["iterations"] for h in e2e_hist))
    e2e_value = world * K / ranks.max_over_ranks(e2e_s, dist, dev)
    h2d = 24 * n

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_reference(budget_s=30.0, max_steps=K)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(K, world),
            "algorithm": f"warm start {headline} (the reference's p = 0 is warm_start_modes.zero)",
            "warm_start": headline,
            "warm_start_modes": modes,
            "speedup_vs_plain": value / (world * modes["zero"]["steps_per_s"]) if modes.get("zero") else None,
            "particle_updates_per_s": value * n,
            "jacobi_iterations_mean": float(np.mean(iters)), "avg_err_max": float(np.max([h["avg_err"] for h in hist])),
            "v_max_max": float(np.max([h["v_max"] for h in hist])),
            "n_ff_pairs_mean": float(np.mean([h["n_ff_pairs"] for h in hist])),
            "phase_ms_mean": {"front": float(np.mean(t_front)), "warm_start": float(np.mean(t_warm)),
                              "jacobi": float(np.mean(t_jac))},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_jacobi (persistent solve + kick/drift)",
                         "bytes_rule": "per launch: iterations * (100 N + 8 P_ff) + 112 N"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": 24 * n + 80, "jacobi_iterations": e2e_iters,
                    "call": "sph_update_fluid + sph_step + sph_get_fluid per step"},
            "gpu_launches": kernels_per_step(headline) * K,
            "clocks": clock,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def bench_batched(args):
    """64 independent dam breaks (log-uniform 5k-200k particles) advanced in
    one batch, launch shapes from the autotuner, versus the same scenes solved
    one context at a time.  Under torchrun the scenes are sharded over the
    ranks by particle count (strong scaling: the 64-scene step is the unit);
    the step time is the slowest rank's.  Prints its own JSON line."""
    import torch

    from warpsph_b200 import autotune as at
    from warpsph_b200 import ranks
    from warpsph_b200.batch import BatchIISPH
    from warpsph_b200.params import SolverParams
    from warpsph_b200.scenes import batched_scenes
    from warpsph_b200.solver import IISPH

    rank, world, local = ranks.env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = ranks.init("nccl", device=dev)
    all_scenes = batched_scenes()
    n_all = sum(s.n for s in all_scenes)
    mine = ranks.partition_scenes([s.n for s in all_scenes], world)[rank]
    scenes = [all_scenes[k] for k in mine]
    n = sum(s.n for s in scenes)
    params = SolverParams(diameter=0.01, gravity=9.81, w_table_size=1024, g_table_size=1024,
                          device=local, **warm_kwargs(args.warm))
    tuned = at.autotune(scenes, params, warm=10, steps=10)
    tp = at.apply(params, tuned)
    K = args.steps
    b = BatchIISPH(scenes, tp)
    b.prepare()
    if args.warmup:
        b.steps(args.warmup)
    b.close()
    b = BatchIISPH(scenes, tp)  # timed from the scenes' initial states
    b.prepare()
    st = torch.cuda.ExternalStream(b._lib.sph_stream(b._ctx), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0.record(st)
    rc = b._lib.sph_launch_steps(b._ctx, K)
    e1.record(st)
    e1.synchronize()
    clock = clocks.stop()
    if rc != 0:
        raise RuntimeError(f"sph_launch_steps failed ({rc})")
    ms = ranks.max_over_ranks(e0.elapsed_time(e1), dist, dev)
    stats = b.scene_stats()
    b.close()
    # the same scenes, one context each, K steps each
    seq_ms = 0.0
    for sc in scenes:
        s = IISPH(stage_path=None, params=tp, scene=sc)
        s._lib.sph_prepare(s._ctx)
        sst = torch.cuda.ExternalStream(s._lib.sph_stream(s._ctx), device=dev)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a0.record(sst)
        s._lib.sph_launch_steps(s._ctx, K)
        a1.record(sst)
        a1.synchronize()
        seq_ms += a0.elapsed_time(a1)
        s.close()
    seq_ms = ranks.max_over_ranks(seq_ms, dist, dev)
    if rank == 0:
        line = {"metric": "batched IISPH steps/s (64 scenes per step)", "value": K / (ms / 1000.0),
                "unit": "steps/s", "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": ms / K,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": f"64 dam breaks, {n_all} fluid particles in total, steps [0, {K})",
                           "warm_start": args.warm, "parallelism": f"scenes sharded over {world}"},
                "particle_updates_per_s": n_all * K / (ms / 1000.0),
                "sequential_contexts_steps_per_s": K / (seq_ms / 1000.0),
                "batch_speedup": seq_ms / ms, "autotuned_rank0": {k: v for k, v in tuned.items() if k != "trials"},
                "last_step_iterations_rank0": {"min": int(stats["iterations"].min()),
                                               "max": int(stats["iterations"].max())},
                "clocks": clock}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def bench_pour(args):
    """The pour onto a procedural obstacle (warpsph_b200.pour): the inlet
    emits layers until 2,000,000 fluid particles have entered (untimed, device
    appends between step batches), then K steps are timed with the emitter off
    (CUDA events on the library's stream).  Prints its own JSON line."""
    import torch

    from warpsph_b200 import _lib, pour

    dev = torch.device("cuda", 0)
    sol, inlet = pour.make(**warm_kwargs(args.warm))
    t0 = time.perf_counter()
    emit_steps = pour.emit_until(sol, inlet)
    emit_s = time.perf_counter() - t0
    if args.warmup:
        sol.steps(args.warmup)
    _lib.check(sol._ctx, sol._lib.sph_prepare(sol._ctx))
    st = torch.cuda.ExternalStream(sol._lib.sph_stream(sol._ctx), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    e0.record(st)
    _lib.check(sol._ctx, sol._lib.sph_launch_steps(sol._ctx, args.steps))
    e1.record(st)
    e1.synchronize()
    clock = clocks.stop()
    ms = e0.elapsed_time(e1)
    hist = sol.stats_history(args.steps)
    flags = 0
    for h in hist:
        flags |= h["flags"]
    if flags & (_lib.SPH_F_TIMEOUT | _lib.SPH_F_NONFINITE | _lib.SPH_F_FF_OVERFLOW | _lib.SPH_F_FB_OVERFLOW):
        raise RuntimeError(f"step flags {flags:#x} in the timed region")
    line = {"metric": "IISPH steps/s, 2M-particle pour onto a procedural obstacle", "value": args.steps / (ms / 1e3),
            "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"pour: {sol.n} fluid + {sol.boundary_n} boundary particles, 0.008 m, "
                                   f"steps after emission ended", "warm_start": args.warm},
            "particle_updates_per_s": sol.n * args.steps / (ms / 1e3),
            "jacobi_iterations_mean": float(np.mean([h["iterations"] for h in hist])),
            "n_ff_pairs_mean": float(np.mean([h["n_ff_pairs"] for h in hist])),
            "v_max_max": float(max(h["v_max"] for h in hist)),
            "emission": {"steps": emit_steps, "wall_s": emit_s, "sim_time": sol.sim_time},
            "clocks": clock}
    sol.close()
    print(json.dumps(line), flush=True)


def bench_solve_shapes(args):
    """k_jacobi alone on the 1M dam break at 10 fixed Jacobi iterations, for
    each launch shape in --solve-shapes (threads,particles per thread,unroll):
    CUDA events around the solve launch on the library's stream, median over
    args.steps steps after 2 discarded ones.  One JSON line per shape."""
    import torch

    from warpsph_b200 import _lib
    from warpsph_b200.params import preset_params
    from warpsph_b200.scenes import preset_scene
    from warpsph_b200.solver import IISPH

    scene = preset_scene(PRESET)
    dev = torch.device("cuda", 0)
    steps = max(3, args.steps)
    for shape in args.solve_shapes.split():
        T, P, U = (int(v) for v in shape.split(","))
        s = IISPH(stage_path=None, params=preset_params(PRESET, device=0, fixed_iters=10, warm_start="zero",
                                                          jacobi_block=T, jacobi_ppt=P, jacobi_unroll=U), scene=scene)
        st = torch.cuda.ExternalStream(s._lib.sph_stream(s._ctx), device=dev)
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps + 2)]
        torch.cuda.synchronize()
        for e in ev:
            _lib.check(s._ctx, s._lib.sph_launch_phase(s._ctx, 0))
            e[0].record(st)
            _lib.check(s._ctx, s._lib.sph_launch_phase(s._ctx, 3))
            e[1].record(st)
        torch.cuda.synchronize()
        t = sorted(e[0].elapsed_time(e[1]) for e in ev[2:])
        h = s.stats_history(steps + 2)[-1]
        s.close()
        med = t[len(t) // 2]
        byts = 10 * (100.0 * scene.n + 8.0 * h["n_ff_pairs"]) + 112.0 * scene.n
        print(json.dumps({"solve_shape": [T, P, U], "ms": med, "us_per_iteration": med * 100.0,
                          "GBps": byts / (med / 1e3) / 1e9, "iterations": h["iterations"]}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)  # the 1M dam break's 500-step run
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true", help="only warm-up + K steps (for ncu captures)")
    ap.add_argument("--workload", choices=["dam_break_1m", "batched64", "pour_2m"], default="dam_break_1m")
    ap.add_argument("--solve-shapes", default="",
                    help="time k_jacobi alone (10 fixed iterations) for these launch shapes, e.g. "
                         "'256,1,4 256,1,2' (threads,particles per thread,unroll)")
    ap.add_argument("--warm", choices=["zero", "half", "mlp", "mlp_continue"], default=None,
                    help="warm start of the headline run: mlp_continue = learned, continuing from a solve "
                         "that stopped at the iteration cap (default for the dam break), mlp = learned "
                         "(default for the batch), zero = the reference's p <- 0 (default for the pour, "
                         "whose splashes lie outside the network's dam-break training data), half = 0.5 p_prev")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.warm is None:
        args.warm = {"pour_2m": "zero", "batched64": "mlp"}.get(args.workload, "mlp_continue")
    if args.impl == "reference":
        bench_reference(args)
    elif args.solve_shapes:
        bench_solve_shapes(args)
    elif args.workload == "batched64":
        bench_batched(args)
    elif args.workload == "pour_2m":
        bench_pour(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
