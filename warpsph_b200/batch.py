"""Batched solving: many independent scenes advanced together in one launch
sequence per step (one sort, one neighbour build, one persistent Jacobi solve).

Each scene keeps its own grid, dt, CFL, residual, convergence decision and
iteration count; scenes that converge drop out of the remaining Jacobi passes
while the others iterate.  Results per scene are identical to solving that
scene alone (same grid, same sorted order, same chunk partition).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .params import SolverParams
from .scenes import Scene


class BatchIISPH:
    def __init__(self, scenes: list[Scene], params: SolverParams, mlp_blob=None):
        self.scenes = scenes
        self.params = params
        self.S = len(scenes)
        self._lib = _lib.load()
        descs = (_lib.SphSceneDesc * self.S)()
        self._keep = []
        for k, sc in enumerate(scenes):
            x = np.ascontiguousarray(sc.fluid_x, np.float32)
            v = np.ascontiguousarray(sc.fluid_v, np.float32)
            b = np.ascontiguousarray(sc.boundary_x, np.float32)
            self._keep += [x, v, b]
            descs[k].x3, descs[k].v3, descs[k].n = x.ctypes.data, v.ctypes.data, len(x)
            descs[k].xb3, descs[k].vb3, descs[k].nb = b.ctypes.data, None, len(b)
        cp = params.to_c()
        ctx = ctypes.c_void_p()
        rc = self._lib.sph_create_batch(ctypes.byref(cp), descs, self.S, ctypes.byref(ctx))
        if rc != _lib.SPH_OK:
            raise _lib.SphError(rc, "sph_create_batch failed")
        self._ctx = ctx
        if params.warm_start == "mlp":
            from .learned import load_blob

            blob = load_blob() if mlp_blob is None else np.ascontiguousarray(mlp_blob, np.float32)
            _lib.check(ctx, self._lib.sph_set_mlp(ctx, _lib.ptr(blob), len(blob)))
        self.fluid_off = np.zeros(self.S + 1, np.int64)
        self.boundary_off = np.zeros(self.S + 1, np.int64)
        _lib.check(ctx, self._lib.sph_get_scene_ranges(ctx, _lib.ptr(self.fluid_off), _lib.ptr(self.boundary_off)))
        self.n = int(self.fluid_off[-1])
        self.last_stats = None

    def prepare(self):
        _lib.check(self._ctx, self._lib.sph_prepare(self._ctx))

    def step(self):
        st = _lib.SphStepStats()
        rc = self._lib.sph_step(self._ctx, ctypes.byref(st))
        self.last_stats = st.as_dict()
        _lib.check(self._ctx, rc)

    def steps(self, count: int):
        st = _lib.SphStepStats()
        rc = self._lib.sph_steps(self._ctx, int(count), ctypes.byref(st))
        self.last_stats = st.as_dict()
        _lib.check(self._ctx, rc)

    def scene_stats(self) -> dict:
        it = np.zeros(self.S, np.int32)
        err, vmax, dt, t = (np.zeros(self.S) for _ in range(4))
        _lib.check(self._ctx, self._lib.sph_get_scene_stats(self._ctx, _lib.ptr(it), _lib.ptr(err), _lib.ptr(vmax),
                                                            _lib.ptr(dt), _lib.ptr(t)))
        return {"iterations": it, "avg_err": err, "v_max": vmax, "dt": dt, "sim_time": t}

    def fluid(self):
        """(x, v, p) of all scenes, concatenated in scene order."""
        x = np.zeros((self.n, 3), np.float32)
        v = np.zeros((self.n, 3), np.float32)
        p = np.zeros(self.n, np.float32)
        _lib.check(self._ctx, self._lib.sph_get_fluid(self._ctx, _lib.ptr(x), _lib.ptr(v), _lib.ptr(p), None, None))
        return x, v, p

    def scene_fluid(self, k: int):
        x, v, p = self.fluid()
        a, b = self.fluid_off[k], self.fluid_off[k + 1]
        return x[a:b], v[a:b], p[a:b]

    def close(self):
        if self._ctx is not None:
            self._lib.sph_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
