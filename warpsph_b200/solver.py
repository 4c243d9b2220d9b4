"""Drop-in replacement of ``wp_sph.solver.IISPH`` (wp_sph/solver/IISPH.py:736-1501).

Same constructor, methods (``step``, ``render``, ``neighbor_search``,
``init_particles``), properties (``average_rho_error``, ``window_closed``) and
attributes (``x v p rho rho_adv n boundary_x boundary_v boundary_phi boundary_n
boundary_hide_n dt inv_dt sim_time``, ``term_d_ii term_a_ii sum_d_ij_p_j v_adv
term_Ap_i``).  Array attributes are device-resident views whose ``.numpy()``
returns the field in original particle order, like ``wp.array.numpy()``.

All computation runs in libwpsph.so on one CUDA device; there is no CPU path.
"""

from __future__ import annotations

import ctypes
import importlib
import warnings

import numpy as np

from . import _lib
from .frames import FrameRecorder
from .params import SolverParams
from .scenes import Scene, box_scene
from .tables import kernel_tables


class DeviceField:
    """A solver field living on the GPU; ``.numpy()`` copies it back in original order."""

    def __init__(self, solver: "IISPH", name: str, width: int, count: str):
        self._solver, self._name, self._width, self._count = solver, name, width, count

    def numpy(self) -> np.ndarray:
        return self._solver._fetch(self._name)

    @property
    def shape(self):
        n = getattr(self._solver, self._count)
        return (n, self._width) if self._width > 1 else (n,)

    def __len__(self):
        return getattr(self._solver, self._count)

    def __array__(self, dtype=None, copy=None):
        a = self.numpy()
        return a if dtype is None else a.astype(dtype)

    def __repr__(self):
        return f"DeviceField({self._name}, shape={self.shape})"


def _reference_constants():
    try:
        return importlib.import_module("wp_sph.main")
    except ImportError:  # package used without the wp_sph shim
        return None


class IISPH:
    def __init__(self, stage_path="example_sph.usd", preview=False, verbose=False, *,
                 params: SolverParams | None = None, scene: Scene | None = None):
        self.verbose = verbose
        main = _reference_constants()
        if params is None:
            params = SolverParams.from_reference_module(main) if main is not None else SolverParams()
        self.params = params
        self._fps = getattr(main, "FPS", 60)
        box = (getattr(main, "BOX_WIDTH", 4.0), getattr(main, "BOX_HEIGHT", 4.0), getattr(main, "BOX_LENGTH", 4.0))
        self._box = box

        # render params (IISPH.py:741-744)
        self.frame_dt = 1.0 / self._fps
        self.sim_time = 0.0
        self.last_frame_time = 0.0
        # simulation params (IISPH.py:746-749)
        self.dt = params.dt_max if params.dt0 is None else params.dt0
        self.inv_dt = 1 / self.dt
        self.boundary_layer = 3
        self.last_stats: dict | None = None
        self._ctx = None
        self._lib = _lib.load()

        rigid_v = None
        if scene is None:
            # IISPH.py:749-766: the fluid block of each scene type
            stype = getattr(main, "scene_type", None)
            name = getattr(stype, "name", "EMPTY")
            bw, bh, bl = box
            layers = 3
            if name == "HOUSE":
                min_point, max_point = (bw * 0.7, bh * 0.01, bl * 0.8), (bw * 0.99, bh * 0.5, bl * 0.99)
            elif name == "PLANE":
                min_point, max_point = (bw * 0.45, bh * 0.05, bl * 0.05), (bw * 0.55, bh * 0.95, bl * 0.95)
                layers = 0
            elif name == "HAND":
                min_point, max_point = (bw * 0.48, bh * 0.05, bl * 0.48), (bw * 0.52, bh * 0.99, bl * 0.52)
            else:
                min_point, max_point = (bw * 0.02, bh * 0.02, bl * 0.02), (bw * 0.98, bh * 0.4, bl * 0.55)
            self.init_particles(min_point, max_point, boundary_layers=layers)
            models = getattr(main, "SCENE_MODELS", {}).get(stype, []) if main is not None else []
            if models:
                self._add_models(models)
            rigid_v = getattr(main, "RIGID_VELOCITY", {}).get(stype) if main is not None else None
            if rigid_v is not None:
                # the rigid body moves (DYNAMIC_SCENE, main.py:20; update_rigid_x, IISPH.py:1356-1365)
                self.params = params = params.replace(move_boundary=True)
        else:
            self._set_scene(scene)

        self._create_context()

        self.renderer = FrameRecorder(stage_path, self._fps) if stage_path else None
        if preview:
            warnings.warn("OpenGL preview is unavailable (no graphics stack); continuing headless")
        self.previewer = None

        self.x = DeviceField(self, "x", 3, "n")
        self.v = DeviceField(self, "v", 3, "n")
        self.p = DeviceField(self, "p", 1, "n")
        self.rho = DeviceField(self, "rho", 1, "n")
        self.rho_adv = DeviceField(self, "rho_adv", 1, "n")
        self.v_adv = DeviceField(self, "v_adv", 3, "n")
        self.term_d_ii = DeviceField(self, "d_ii", 3, "n")
        self.term_a_ii = DeviceField(self, "a_ii", 1, "n")
        self.sum_d_ij_p_j = DeviceField(self, "s", 3, "n")
        self.term_Ap_i = DeviceField(self, "Ap", 1, "n")
        self.boundary_x = DeviceField(self, "boundary_x", 3, "boundary_n")
        self.boundary_phi = DeviceField(self, "boundary_phi", 1, "boundary_n")
        if rigid_v is not None:
            # set_rigid_v at sim_time 0 (IISPH.py:1061-1081), before the first step
            self.set_rigid_velocity(rigid_v)

    # ------------------------------------------------------------------ scene

    def init_particles(self, min_point=None, max_point=None, spacing=None, fluid_depth=0.0, boundary_layers=3):
        """IISPH.init_particles (IISPH.py:857-1000), EMPTY scene type."""
        spacing = self.params.diameter if spacing is None else spacing
        scene = box_scene(self._box, spacing, min_point, max_point, fluid_depth, boundary_layers)
        self._set_scene(scene)
        if self._ctx is not None:
            self._upload()
        print(f"Initialized {self.n} fluid and {self.boundary_n} boundary particles")

    def _add_models(self, models):
        """Mesh models sampled into rigid boundary particles after the box
        walls (IISPH.py:945-991, model.py:53-60)."""
        from .model import load_model

        pts = [load_model(f, scale, np.asarray(pos, np.float64), np.asarray(rot, np.float64),
                          spacing=self.params.diameter, device=self.params.device)
               for f, scale, pos, rot in models]
        for f, p in zip(models, pts):
            print(f"Loaded model {f[0]} with {len(p)} particles")
        s = self._scene
        bx = np.concatenate([s.boundary_x] + [np.asarray(p, np.float32) for p in pts]).astype(np.float32)
        self._set_scene(Scene(s.fluid_x, s.fluid_v, bx, s.boundary_hide_n, s.box))

    def _set_scene(self, scene: Scene):
        self._scene = scene
        self.n = scene.n
        self.boundary_n = scene.boundary_n
        self.boundary_hide_n = scene.boundary_hide_n
        self._boundary_v = np.zeros_like(scene.boundary_x)

    @property
    def boundary_v(self):
        return self._boundary_v

    def set_state(self, x, v=None):
        """Replace fluid positions/velocities (original order) on the device."""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
        v = np.zeros_like(x) if v is None else np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3)
        self._scene = Scene(x, v, self._scene.boundary_x, self._scene.boundary_hide_n, self._scene.box)
        self.n = len(x)
        _lib.check(self._ctx, self._lib.sph_set_fluid(self._ctx, _lib.ptr(x), _lib.ptr(v), self.n))

    def update_state(self, x, v, p=None):
        """Replace positions, velocities and pressures (original order) of the
        current particles, keeping dt, time and the solver's history
        (sph_update_fluid); set_state instead starts a new state.  p=None
        keeps the pressures on the device."""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
        v = np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3)
        pp = None
        if p is not None:
            p = np.ascontiguousarray(p, dtype=np.float32).reshape(-1)
            pp = _lib.ptr(p)
        _lib.check(self._ctx, self._lib.sph_update_fluid(self._ctx, _lib.ptr(x), _lib.ptr(v), pp, len(x)))

    def add_fluid(self, x, v=None):
        """Append fluid particles (e.g. an emitter's new layer) to the state on
        the device.  Existing particles keep their state; new ones start with
        p = 0 and take the next original ids.  No counterpart in the reference,
        whose particle set is fixed at init_particles."""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
        if len(x) == 0:
            return
        v = None if v is None else np.ascontiguousarray(v, dtype=np.float32).reshape(-1, 3)
        _lib.check(self._ctx, self._lib.sph_add_fluid(self._ctx, _lib.ptr(x), _lib.ptr(v), len(x)))
        self.n += len(x)

    def set_boundary_velocity(self, vb):
        """Boundary particle velocities (original order).  Re-uploads the
        boundary at its current positions, which recomputes psi there."""
        self._boundary_v = np.ascontiguousarray(vb, dtype=np.float32).reshape(-1, 3)
        b = np.ascontiguousarray(self.boundary_x.numpy(), dtype=np.float32)
        _lib.check(self._ctx, self._lib.sph_set_boundary(self._ctx, _lib.ptr(b), _lib.ptr(self._boundary_v),
                                                         self.boundary_n))

    def set_rigid_velocity(self, v, start=None):
        """set_rigid_v (IISPH.py:651-659): boundary particles [start, boundary_n)
        (default: those after the box walls, boundary_hide_n) get velocity v.
        With params.move_boundary they move by v dt after every step
        (update_rigid_x, IISPH.py:662-671) and the boundary grid is rebuilt every
        step.  The reference sets the velocity during its first step; call this
        before the first step, so psi stays the one computed at start
        (IISPH.py:811-821)."""
        start = self.boundary_hide_n if start is None else int(start)
        vb = self._boundary_v.copy()
        vb[start:] = np.asarray(v, dtype=np.float32)
        self.set_boundary_velocity(vb)

    def _create_context(self):
        cp = self.params.to_c()
        cp.dt0 = self.dt
        ctx = ctypes.c_void_p()
        rc = self._lib.sph_create(ctypes.byref(cp), ctypes.byref(ctx))
        if rc != _lib.SPH_OK:
            raise _lib.SphError(rc, "sph_create failed (is a CUDA device visible?)")
        self._ctx = ctx
        w, g = kernel_tables(self.params)
        _lib.check(ctx, self._lib.sph_set_tables(ctx, _lib.ptr(w), len(w), _lib.ptr(g), len(g)))
        if self.params.warm_start == "mlp":
            self.set_mlp(self.params.extra.get("mlp_blob"))
        self._upload()

    def set_mlp(self, blob=None):
        """Install the learned warm-start network (default: the shipped weights)."""
        from .learned import load_blob

        blob = load_blob() if blob is None else np.ascontiguousarray(blob, dtype=np.float32)
        _lib.check(self._ctx, self._lib.sph_set_mlp(self._ctx, _lib.ptr(blob), len(blob)))

    def _upload(self):
        s = self._scene
        b = np.ascontiguousarray(s.boundary_x, dtype=np.float32)
        bv = np.ascontiguousarray(self._boundary_v, dtype=np.float32)
        _lib.check(self._ctx, self._lib.sph_set_boundary(self._ctx, _lib.ptr(b), _lib.ptr(bv), len(b)))
        x = np.ascontiguousarray(s.fluid_x, dtype=np.float32)
        v = np.ascontiguousarray(s.fluid_v, dtype=np.float32)
        _lib.check(self._ctx, self._lib.sph_set_fluid(self._ctx, _lib.ptr(x), _lib.ptr(v), len(x)))

    def close(self):
        if self._ctx is not None:
            self._lib.sph_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ stepping

    def step(self):
        """IISPH.step() (IISPH.py:1002-1371): one time step on the GPU."""
        st = _lib.SphStepStats()
        rc = self._lib.sph_step(self._ctx, ctypes.byref(st))
        self._absorb(st)
        _lib.check(self._ctx, rc)

    def steps(self, count: int):
        """``count`` steps with a single host synchronisation."""
        st = _lib.SphStepStats()
        rc = self._lib.sph_steps(self._ctx, int(count), ctypes.byref(st))
        self._absorb(st)
        _lib.check(self._ctx, rc)

    def _absorb(self, st: _lib.SphStepStats):
        self.last_stats = st.as_dict()
        if st.step_index:
            self.sim_time = st.sim_time
            self.dt = st.dt_next
            self.inv_dt = 1 / self.dt
        if st.flags & _lib.SPH_F_NOT_CONVERGED:
            # IISPH.py:1204-1206
            print(f"Pressure solver did not converge at {st.sim_time - st.dt:.2f}s")

    def stats_history(self, count: int) -> list[dict]:
        arr = (_lib.SphStepStats * count)()
        _lib.check(self._ctx, self._lib.sph_get_stats_history(self._ctx, arr, count))
        return [a.as_dict() for a in arr]

    def neighbor_search(self):
        """IISPH.neighbor_search() (IISPH.py:1408-1482)."""
        _lib.check(self._ctx, self._lib.sph_neighbor_search(self._ctx))

    def get_neighbors(self, with_boundary: bool = False):
        """Neighbour sets of the last build as CSR in original ids, ascending."""
        n = self.n
        last = self.last_stats or {}
        cap = max(1, n * max(self.params.max_ff, int(last.get("max_ff_count", 0)) + 1) * 2)
        ff_off = np.zeros(n + 1, np.int64)
        ff_idx = np.zeros(cap, np.int32)
        fb_off = fb_idx = None
        if with_boundary:
            fb_off = np.zeros(n + 1, np.int64)
            fb_idx = np.zeros(cap, np.int32)
        _lib.check(self._ctx, self._lib.sph_get_neighbors(
            self._ctx, _lib.ptr(ff_off), _lib.ptr(ff_idx), cap, _lib.ptr(fb_off), _lib.ptr(fb_idx), cap))
        out = {"ff_off": ff_off, "ff_idx": ff_idx[: ff_off[-1]].copy()}
        if with_boundary:
            out.update(fb_off=fb_off, fb_idx=fb_idx[: fb_off[-1]].copy())
        return out

    def set_dt(self, dt: float, inv_dt: float | None = None):
        inv_dt = 1.0 / dt if inv_dt is None else inv_dt
        _lib.check(self._ctx, self._lib.sph_set_dt(self._ctx, float(dt), float(inv_dt)))
        self.dt, self.inv_dt = dt, inv_dt

    def set_pressure(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _lib.check(self._ctx, self._lib.sph_set_pressure(self._ctx, _lib.ptr(p), len(p)))

    # ------------------------------------------------------------------ readback

    def _fetch(self, name: str) -> np.ndarray:
        n, nb = self.n, self.boundary_n
        if name in ("x", "v", "p", "rho", "rho_adv"):
            out = np.zeros((n, 3) if name in ("x", "v") else (n,), np.float32)
            args = {k: None for k in ("x", "v", "p", "rho", "rho_adv")}
            args[name] = out
            _lib.check(self._ctx, self._lib.sph_get_fluid(self._ctx, *(_lib.ptr(args[k]) for k in
                                                                       ("x", "v", "p", "rho", "rho_adv"))))
            return out
        if name in ("d_ii", "a_ii", "s", "v_adv", "Ap"):
            out = np.zeros((n, 3) if name in ("d_ii", "s", "v_adv") else (n,), np.float32)
            args = {k: None for k in ("d_ii", "a_ii", "s", "v_adv", "Ap")}
            args[name] = out
            _lib.check(self._ctx, self._lib.sph_get_terms(self._ctx, *(_lib.ptr(args[k]) for k in
                                                                       ("d_ii", "a_ii", "s", "v_adv", "Ap"))))
            return out
        if name in ("boundary_x", "boundary_phi"):
            out = np.zeros((nb, 3) if name == "boundary_x" else (nb,), np.float32)
            xb = out if name == "boundary_x" else None
            ph = out if name == "boundary_phi" else None
            _lib.check(self._ctx, self._lib.sph_get_boundary(self._ctx, _lib.ptr(xb), _lib.ptr(ph)))
            return out
        raise KeyError(name)

    # ------------------------------------------------------------------ reference surface

    @property
    def average_rho_error(self):
        """IISPH.average_rho_error (IISPH.py:1489-1494), FP64 on the device."""
        return 0.0 if self.last_stats is None else self.last_stats["avg_err"]

    @property
    def window_closed(self):
        return False

    def render(self):
        """IISPH.render (IISPH.py:1396-1406), headless: records positions at FPS."""
        if self.renderer is None:
            return
        if self.sim_time - self.last_frame_time >= self.frame_dt:
            rigid = self.boundary_x.numpy()[self.boundary_hide_n:]
            self.renderer.add(self.sim_time, self.x.numpy(), rigid)
            self.last_frame_time = self.sim_time

    def raise_error(self, message):
        if self.renderer:
            self.renderer.save()
        raise RuntimeError(message)
