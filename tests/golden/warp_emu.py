"""Minimal numpy emulation of the warp-lang 1.7.1 API subset used by the
reference IISPH solver (wp_sph/solver/IISPH.py, wp_sph/solver/sph_funcs.py).

Test infrastructure only: it lets ``make_golden.py`` import and run the
reference's own kernel source in this container, where warp-lang (pinned at
1.7.1 in the reference's uv.lock:217-218) is not installed.  Nothing in the
product imports this file.

Semantics restated from Warp's public documentation:

* ``@wp.kernel`` functions run once per thread id, sequentially in tid order.
  Module-level Python floats referenced from kernel code become float32
  constants (Warp captures them as ``wp.float32``), so the kernel body is
  re-bound to a copy of its globals with floats cast to ``np.float32``.
  Arithmetic then stays in IEEE float32 through NumPy 2's weak-scalar
  promotion, with no fused multiply-add contraction.
* ``wp.length``/``wp.dot`` evaluate ``x*x + y*y + z*z`` left to right in float32.
* ``wp.sign(x)`` is -1 for x < 0 and +1 otherwise.
* ``wp.HashGrid``: cell width = build radius; ``hash_grid_point_id(tid)`` is the
  tid-th point in cell-sorted order; ``hash_grid_query(x, r)`` yields every point
  of the cells overlapping [x-r, x+r]^3, each cell once.  Warp hashes cell
  coordinates modulo the grid dims; callers filter candidates by distance, so the
  filtered neighbour SET does not depend on the hashing, only the visiting order
  does.  This emulation visits the true (unhashed) cells, which yields the same
  filtered sets in a different summation order.
* ``wp.atomic_add``/``wp.atomic_max`` apply in tid order and return the old value.
"""

from __future__ import annotations

import contextlib
import math
import sys
import types

import numpy as np

pi = math.pi
float32 = np.float32
float64 = np.float64
uint64 = np.uint64


def int32(x=0):
    return int(x)


class _VecType:
    length = 3

    def __call__(self, *args):
        if len(args) == 1:
            return np.full(3, args[0], dtype=np.float32)
        return np.array(args, dtype=np.float32)


vec3 = _VecType()


def constant(x):
    return x


# ---------------------------------------------------------------- arrays

class array:
    """Host-resident stand-in for wp.array (float32 / int32 / vec3)."""

    def __init__(self, data=None, dtype=float, shape=None):
        self.dtype = dtype
        if data is None and shape is None:
            self._a = None  # type annotation use: wp.array(dtype=...)
            return
        if data is None:
            data = np.zeros(shape)
        np_dtype, width = _np_layout(dtype)
        a = np.array(data, dtype=np_dtype)
        if width:
            a = a.reshape(-1, width)
        self._a = a

    def __len__(self):
        return self._a.shape[0]

    @property
    def shape(self):
        return (self._a.shape[0],)

    def __getitem__(self, i):
        v = self._a[i]
        if isinstance(v, np.ndarray):
            return v.copy()
        return v

    def __setitem__(self, i, value):
        self._a[i] = value

    def numpy(self):
        return self._a.copy()

    def assign(self, value):
        self._a[...] = np.asarray(value, dtype=self._a.dtype).reshape(self._a.shape)


def _np_layout(dtype):
    if dtype is vec3:
        return np.float32, 3
    if dtype in (int, int32, np.int32):
        return np.int32, 0
    if dtype in (float, float32, np.float32):
        return np.float32, 0
    raise TypeError(f"unsupported dtype {dtype}")


def zeros(n, dtype=float):
    np_dtype, width = _np_layout(dtype)
    shape = (n, width) if width else (n,)
    return array(np.zeros(shape, dtype=np_dtype), dtype=dtype)


def zeros_like(a):
    return array(np.zeros_like(a._a), dtype=a.dtype)


def from_numpy(a, dtype=float):
    return array(a, dtype=dtype)


# ---------------------------------------------------------------- builtins

def length(v):
    return np.sqrt(dot(v, v))


def dot(a, b):
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def normalize(v):
    return v / length(v)


def min(a, b):  # noqa: A001 - mirrors the Warp builtin name
    return a if a < b else b


def max(a, b):  # noqa: A001
    return a if a > b else b


def abs(x):  # noqa: A001
    return np.abs(x)


def sign(x):
    return np.float32(-1.0) if x < 0 else np.float32(1.0)


def atomic_add(arr, idx, value):
    old = arr[idx]
    arr[idx] = old + value
    return old


def atomic_max(arr, idx, value):
    old = arr[idx]
    if value > old:
        arr[idx] = value
    return old


# ---------------------------------------------------------------- hash grid

_GRIDS: dict[int, "HashGrid"] = {}


class HashGrid:
    def __init__(self, dim_x, dim_y, dim_z):
        if dim_x < 1 or dim_y < 1 or dim_z < 1:
            raise ValueError("HashGrid dims must be >= 1")
        self.dims = (dim_x, dim_y, dim_z)
        self.id = id(self)
        _GRIDS[self.id] = self
        self.point_ids = np.zeros(0, dtype=np.int64)

    def build(self, points, radius):
        pts = points._a.astype(np.float32)
        self.points = pts
        self.radius = np.float32(radius)
        inv = np.float32(1.0) / np.float32(radius)
        cells = np.floor(pts * inv).astype(np.int64)
        self.cells = cells
        dx, dy, dz = self.dims
        hashed = (np.mod(cells[:, 2], dz) * dy + np.mod(cells[:, 1], dy)) * dx + np.mod(cells[:, 0], dx)
        self.point_ids = np.argsort(hashed, kind="stable")
        table: dict[tuple, list] = {}
        for p in self.point_ids:
            table.setdefault(tuple(cells[p]), []).append(int(p))
        self.table = table


def hash_grid_point_id(grid_id, tid):
    return int(_GRIDS[grid_id].point_ids[tid])


def hash_grid_query(grid_id, x, radius):
    g = _GRIDS[grid_id]
    inv = np.float32(1.0) / g.radius
    r = np.float32(radius)
    lo = np.floor((np.asarray(x, np.float32) - r) * inv).astype(np.int64)
    hi = np.floor((np.asarray(x, np.float32) + r) * inv).astype(np.int64)
    for cz in range(lo[2], hi[2] + 1):
        for cy in range(lo[1], hi[1] + 1):
            for cx in range(lo[0], hi[0] + 1):
                yield from g.table.get((cx, cy, cz), ())


# ---------------------------------------------------------------- kernels

_FUNC_MARK = "__warp_emu_func__"


def func(f):
    setattr(f, _FUNC_MARK, True)
    return f


def _rebind(f, cache):
    """Copy ``f`` with float globals cast to float32 (kernel constant semantics)."""
    if f in cache:
        return cache[f]
    g = {}
    new = types.FunctionType(f.__code__, g, f.__name__, f.__defaults__, f.__closure__)
    cache[f] = new
    for k, v in f.__globals__.items():
        if isinstance(v, float):
            g[k] = np.float32(v)
        elif isinstance(v, types.FunctionType) and getattr(v, _FUNC_MARK, False):
            g[k] = _rebind(v, cache)
        else:
            g[k] = v
    return new


class _Kernel:
    def __init__(self, f):
        self.f = f
        self.__name__ = f.__name__


def kernel(f):
    return _Kernel(f)


_TID = [0]


def tid():
    return _TID[0]


def launch(kernel, dim, inputs=(), outputs=(), device=None):
    f = _rebind(kernel.f, {})
    ann = kernel.f.__annotations__
    names = kernel.f.__code__.co_varnames[: kernel.f.__code__.co_argcount]
    args = []
    for name, a in zip(names, list(inputs) + list(outputs)):
        t = ann.get(name)
        if t is float:
            a = np.float32(a)
        elif t is int:
            a = int(a)
        elif t is vec3:
            a = np.asarray(a, dtype=np.float32)
        args.append(a)
    for t in range(dim):
        _TID[0] = t
        f(*args)


@contextlib.contextmanager
def ScopedTimer(name, active=False, **kw):
    yield


@contextlib.contextmanager
def ScopedDevice(device=None):
    yield


def install():
    """Register this module as ``warp`` (and a stub ``warp.render``)."""
    mod = sys.modules[__name__]
    render = types.ModuleType("warp.render")

    class _NoRenderer:
        def __init__(self, *a, **k):
            raise RuntimeError("rendering is not emulated")

    render.UsdRenderer = _NoRenderer
    render.OpenGLRenderer = _NoRenderer
    mod.render = render
    sys.modules["warp"] = mod
    sys.modules["warp.render"] = render
