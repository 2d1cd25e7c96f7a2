"""A minimal NumPy stand-in for the NVIDIA Warp runtime (`warp-lang`), used only
to execute the reference's own kernel source on the CPU when generating golden
fixtures (`tests/golden/make_golden.py`).  Warp itself is not installable here.

Semantics restated from Warp's public API documentation:

* `@wp.kernel` functions run once per thread id in `range(dim)`, serially, with
  `wp.tid()` returning the current id (Warp's CPU device also runs a launch's
  threads one after another);
* `float` kernel arguments and `wp.vec3` values are FP32; Python float literals
  combine with FP32 values as FP32 (NumPy's weak-scalar promotion);
* `wp.atomic_add/sub/max` update an array element in place (serial here, so
  thread order);
* tile reductions (`wp.tile`, `wp.tile_sum`, `wp.tile_atomic_add`) reduce to a
  per-thread atomic add;
* `wp.HashGrid` yields every particle of the cells overlapping the query
  sphere; a kernel filters by distance, so the candidate order is the only
  difference from Warp's hash grid (it matters only when a neighbour cache
  overflows).
"""
from __future__ import annotations

import inspect
import math

import numpy as np

f32 = np.float32

float32 = f32
float64 = np.float64
int32 = np.int32
uint32 = np.uint32
int64 = np.int64
uint64 = np.uint64
uint8 = np.uint8
bool = bool  # noqa: A001

_TID = [0]


# --------------------------------------------------------------------- types

class _VecType:
    def __init__(self, n, name):
        self.n = n
        self.__name__ = name

    def __call__(self, *args):
        if len(args) == 0:
            return np.zeros(self.n, dtype=f32)
        if len(args) == 1:
            a = np.asarray(args[0], dtype=f32)
            if a.ndim == 0:
                return np.full(self.n, a, dtype=f32)
            return a.astype(f32).copy()
        return np.array([f32(a) for a in args], dtype=f32)


class Mat(np.ndarray):
    """Square FP32 matrix value: `M * v` is the matrix-vector product and
    `M * N` the matrix product (Warp's operator semantics); with a scalar it
    scales."""

    def _mv(self, v):
        a = np.asarray(self, dtype=f32)
        n = a.shape[0]
        out = np.zeros(n, dtype=f32)
        for r in range(n):
            acc = a[r, 0] * v[0]
            for c in range(1, n):
                acc = acc + a[r, c] * v[c]
            out[r] = acc
        return out

    def __mul__(self, other):
        o = np.asarray(other)
        if o.ndim == 1:
            return self._mv(o.astype(f32))
        if o.ndim == 2:
            return np.stack([self._mv(o[:, c].astype(f32)) for c in range(o.shape[1])], axis=1).view(Mat)
        return np.multiply(np.asarray(self), o).astype(f32).view(Mat)

    def __rmul__(self, other):
        return np.multiply(np.asarray(other), np.asarray(self)).astype(f32).view(Mat)


def _mat(a):
    return np.asarray(a, dtype=f32).copy().view(Mat)


class _MatType:
    def __init__(self, n, name):
        self.n = n
        self.__name__ = name

    def __call__(self, *args):
        if len(args) == 0:
            return _mat(np.zeros((self.n, self.n)))
        if len(args) == self.n * self.n:
            return _mat(np.array([f32(a) for a in args], dtype=f32).reshape(self.n, self.n))
        if len(args) == self.n:
            return _mat(np.stack([np.asarray(a, dtype=f32) for a in args], axis=1))
        return _mat(np.asarray(args[0], dtype=f32).reshape(self.n, self.n))


vec2 = _VecType(2, "vec2")
vec3 = _VecType(3, "vec3")
vec4 = _VecType(4, "vec4")
vec3f = vec3
mat22 = _MatType(2, "mat22")
mat33 = _MatType(3, "mat33")
mat44 = _MatType(4, "mat44")
quat = vec4
transform = _VecType(7, "transform")


def _elem_shape(dtype):
    if isinstance(dtype, _VecType):
        return (dtype.n,), f32
    if isinstance(dtype, _MatType):
        return (dtype.n, dtype.n), f32
    if dtype is float or dtype is f32:
        return (), f32
    if dtype is int or dtype in (np.int32,):
        return (), np.int32
    if dtype in (np.uint64, np.int64):
        return (), np.int64
    if dtype in (np.uint32,):
        return (), np.uint32
    if dtype in (np.uint8, bool):
        return (), np.uint8
    return (), f32


class ShimArray:
    """Device array stand-in backed by a NumPy array."""

    def __init__(self, data: np.ndarray, dtype):
        self.data = data
        self.dtype = dtype

    def __len__(self):
        return self.data.shape[0]

    @property
    def shape(self):
        return (self.data.shape[0],)

    @property
    def size(self):
        return self.data.shape[0]

    def __getitem__(self, idx):
        if isinstance(idx, slice):
            return ShimArray(self.data[idx], self.dtype)
        v = self.data[int(idx)]
        if isinstance(v, np.ndarray):
            return _mat(v) if isinstance(self.dtype, _MatType) else v.copy()
        return v

    def __setitem__(self, idx, val):
        self.data[int(idx)] = val

    def numpy(self):
        return self.data

    def zero_(self):
        self.data[...] = 0

    def fill_(self, v):
        self.data[...] = v

    def assign(self, src):
        self.data[...] = src.data if isinstance(src, ShimArray) else np.asarray(src)

    @property
    def ptr(self):
        return id(self)


def array(data=None, dtype=None, device=None, shape=None, **kw):
    if data is None and shape is None:
        return ("array-type", dtype)  # annotation use: wp.array(dtype=...)
    if data is None:
        n = shape if isinstance(shape, int) else shape[0]
        return zeros(n, dtype=dtype)
    eshape, npdt = _elem_shape(dtype)
    a = np.array(data, dtype=npdt, copy=True)
    if eshape:
        a = a.reshape((-1,) + eshape)
    return ShimArray(a, dtype)


def zeros(n, dtype=float, device=None, **kw):
    if isinstance(n, tuple):
        n = n[0]
    eshape, npdt = _elem_shape(dtype)
    return ShimArray(np.zeros((int(n),) + eshape, dtype=npdt), dtype)


def empty(n, dtype=float, device=None, **kw):
    return zeros(n, dtype=dtype)


def full(n, value, dtype=float, device=None, **kw):
    a = zeros(n, dtype=dtype)
    a.data[...] = value
    return a


def zeros_like(a):
    return ShimArray(np.zeros_like(a.data), a.dtype)


def clone(a):
    return ShimArray(a.data.copy(), a.dtype)


def copy(dest, src, dest_offset=0, src_offset=0, count=None):
    s = src.data if isinstance(src, ShimArray) else np.asarray(src)
    if count is None:
        count = min(len(dest), s.shape[0] - src_offset)
    dest.data[dest_offset:dest_offset + count] = s[src_offset:src_offset + count]


# ------------------------------------------------------------------ runtime

class _Device:
    def __init__(self, name="cpu"):
        self.alias = name
        self.is_cuda = False

    def __str__(self):
        return self.alias


def init():
    pass


def get_device(name=None):
    return _Device()


def set_device(name):
    pass


def synchronize():
    pass


def synchronize_device(*a):
    pass


class ScopedTimer:
    def __init__(self, *a, **k):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def tid():
    return _TID[0]


def func(f=None, **kw):
    if f is None:
        return lambda g: g
    return f


class Kernel:
    def __init__(self, fn):
        self.fn = fn
        self.key = fn.__name__
        sig = inspect.signature(fn)
        self.params = list(sig.parameters.values())

    def run(self, dim, args):
        conv = []
        for p, a in zip(self.params, args):
            ann = p.annotation
            if ann is float and not isinstance(a, ShimArray):
                a = f32(a)
            elif ann is int and not isinstance(a, ShimArray):
                a = int(a)
            elif isinstance(ann, _VecType) and not isinstance(a, ShimArray):
                a = np.asarray(a, dtype=f32).copy()
            conv.append(a)
        fn = self.fn
        n = int(dim[0]) if isinstance(dim, (tuple, list)) else int(dim)
        for t in range(n):
            _TID[0] = t
            fn(*conv)


def kernel(f=None, **kw):
    if f is None:
        return lambda g: Kernel(g)
    return Kernel(f)


def launch(kernel, dim, inputs=(), outputs=(), device=None, block_dim=None, stream=None, **kw):
    kernel.run(dim, list(inputs) + list(outputs))


# -------------------------------------------------------------------- math

def dot(a, b):
    a = np.asarray(a, dtype=f32)
    b = np.asarray(b, dtype=f32)
    s = a[0] * b[0]
    for i in range(1, a.shape[0]):
        s = s + a[i] * b[i]
    return f32(s)


def length(a):
    return f32(np.sqrt(dot(a, a)))


def length_sq(a):
    return dot(a, a)


def normalize(a):
    ln = length(a)
    if ln > 0:
        return (np.asarray(a, dtype=f32) / ln).astype(f32)
    return np.zeros_like(a)


def cross(a, b):
    a = np.asarray(a, dtype=f32)
    b = np.asarray(b, dtype=f32)
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], dtype=f32)


def outer(a, b):
    return _mat(np.outer(np.asarray(a, dtype=f32), np.asarray(b, dtype=f32)))


def inverse(m):
    return _mat(np.linalg.inv(np.asarray(m, dtype=np.float64)))


def determinant(m):
    return f32(np.linalg.det(np.asarray(m, dtype=np.float64)))


def transpose(m):
    return np.asarray(m).T.copy()


def mul(a, b):
    return np.asarray(a) @ np.asarray(b) if np.ndim(a) == 2 else a * b


def max(a, b):  # noqa: A001
    return np.maximum(a, b)


def min(a, b):  # noqa: A001
    return np.minimum(a, b)


def abs(a):  # noqa: A001
    return np.abs(a)


def sqrt(a):
    return f32(np.sqrt(f32(a)))


def exp(a):
    return f32(np.exp(f32(a)))


def log(a):
    return f32(np.log(f32(a)))


def pow(a, b):  # noqa: A001
    return f32(np.power(f32(a), f32(b)))


def sin(a):
    return f32(np.sin(f32(a)))


def cos(a):
    return f32(np.cos(f32(a)))


def acos(a):
    return f32(np.arccos(f32(a)))


def floor(a):
    return f32(np.floor(a))


def clamp(a, lo, hi):
    return np.minimum(np.maximum(a, lo), hi)


def select(cond, a, b):
    return b if cond else a


def where(cond, a, b):
    return a if cond else b


def atomic_add(arr, idx, val):
    arr.data[int(idx)] = arr.data[int(idx)] + val
    return arr.data[int(idx)]


def atomic_sub(arr, idx, val):
    arr.data[int(idx)] = arr.data[int(idx)] - val
    return arr.data[int(idx)]


def atomic_max(arr, idx, val):
    arr.data[int(idx)] = np.maximum(arr.data[int(idx)], val)
    return arr.data[int(idx)]


def atomic_min(arr, idx, val):
    arr.data[int(idx)] = np.minimum(arr.data[int(idx)], val)
    return arr.data[int(idx)]


def tile(val, **kw):
    return val


def tile_sum(t):
    return t


def tile_atomic_add(arr, val, offset=0):
    arr.data[offset] = arr.data[offset] + val


# --------------------------------------------------------------- hash grid

_GRIDS = {}


class HashGrid:
    def __init__(self, dim_x, dim_y, dim_z, device=None):
        self.dims = (int(dim_x), int(dim_y), int(dim_z))
        self.id = len(_GRIDS) + 1
        _GRIDS[self.id] = self
        self.cells = {}
        self.points = None
        self.cell_width = 1.0

    def build(self, points, radius):
        self.points = points.data if isinstance(points, ShimArray) else np.asarray(points)
        self.cell_width = float(radius)
        self.cells = {}
        cw = self.cell_width
        for i, p in enumerate(self.points):
            key = tuple(int(math.floor(float(p[a]) / cw)) for a in range(3))
            self.cells.setdefault(key, []).append(i)


def hash_grid_query(grid_id, point, radius):
    g = _GRIDS[int(grid_id)]
    cw = g.cell_width
    p = [float(point[a]) for a in range(3)]
    lo = [int(math.floor((p[a] - float(radius)) / cw)) for a in range(3)]
    hi = [int(math.floor((p[a] + float(radius)) / cw)) for a in range(3)]
    out = []
    for cz in range(lo[2], hi[2] + 1):
        for cy in range(lo[1], hi[1] + 1):
            for cx in range(lo[0], hi[0] + 1):
                out.extend(g.cells.get((cx, cy, cz), ()))
    return iter(out)


def hash_grid_query_next(query, index):
    raise NotImplementedError


# ------------------------------------------------------------ misc modules

class _Types:
    array = array
    vec3 = vec3


types = _Types()


class _Render:
    def __getattr__(self, name):
        raise ImportError("warp.render is not available in the NumPy stand-in")


render = _Render()

config = type("config", (), {"mode": "release", "verbose": False, "quiet": True})()
