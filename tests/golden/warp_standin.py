"""A minimal stand-in for the parts of NVIDIA Warp that ipc_warp's hot-path
functions use, so those functions can run as plain Python to produce golden
vectors (tests/golden/make_golden.py).  Generation-time only: nothing here is
used by the product or needed on a GPU machine.

Semantics: vectors/matrices are numpy arrays of the scalar dtype (float32 for
the reference's default build), so each arithmetic operation rounds to that
type; dot products are evaluated as ((x0*y0 + x1*y1) + x2*y2); ``@wp.func``
and ``@wp.kernel`` return the plain function; kernels are run by
:func:`launch` which sets ``wp.tid()``.  BVH/mesh queries enumerate every
primitive whose box overlaps the query box (the reference's queries are
conservative, so the accepted pairs do not depend on the hierarchy).
``closest_point_edge_edge`` (a Warp builtin, not in the reference tree) is the
clamped segment-segment method of Ericson, Real-Time Collision Detection
5.1.9.
"""
from __future__ import annotations

import math
import types as _pytypes

import numpy as np

_state = {"tid": 0}


# --------------------------------------------------------------- decorators
def func(f):
    return f


def kernel(f):
    return f


def struct(cls):
    fields = list(getattr(cls, "__annotations__", {}).keys())

    def make(**kw):
        ns = _pytypes.SimpleNamespace(**{k: None for k in fields})
        for k, v in kw.items():
            setattr(ns, k, v)
        return ns

    make.fields = fields
    return make


def tid():
    return _state["tid"]


def launch(fn, n, *args):
    for i in range(n):
        _state["tid"] = i
        fn(*args)


# ------------------------------------------------------------------- types
class _Scalar:
    def __init__(self, dt):
        self.dt = dt

    def __call__(self, v=0.0):
        return self.dt(v)


float32 = np.float32
float64 = np.float64
uint64 = np.uint64


class _Vec:
    def __init__(self, n, dt):
        self.n, self.dt = n, dt

    def __call__(self, *args):
        if len(args) == 0:
            return np.zeros(self.n, self.dt)
        if len(args) == 1:
            a = args[0]
            if np.ndim(a) == 0:
                return np.full(self.n, a, dtype=self.dt)
            return np.array(a, dtype=self.dt)
        return np.array(args, dtype=self.dt)


class _Mat:
    def __init__(self, r, c, dt):
        self.r, self.c, self.dt = r, c, dt

    def __call__(self, *args):
        if len(args) == 0:
            return np.zeros((self.r, self.c), self.dt)
        if len(args) == 1:
            a = args[0]
            if np.ndim(a) == 0:
                return np.full((self.r, self.c), a, dtype=self.dt)
            return np.array(a, dtype=self.dt).reshape(self.r, self.c)
        return np.array(args, dtype=self.dt).reshape(self.r, self.c)


vec2, vec3, vec4 = _Vec(2, np.float32), _Vec(3, np.float32), _Vec(4, np.float32)
vec2d, vec3d, vec4d = _Vec(2, np.float64), _Vec(3, np.float64), _Vec(4, np.float64)
vec2i, vec3i, vec4i = _Vec(2, np.int32), _Vec(3, np.int32), _Vec(4, np.int32)
mat22, mat33, mat44 = _Mat(2, 2, np.float32), _Mat(3, 3, np.float32), _Mat(4, 4, np.float32)
mat22d, mat33d, mat44d = _Mat(2, 2, np.float64), _Mat(3, 3, np.float64), _Mat(4, 4, np.float64)
quat, quatd = _Vec(4, np.float32), _Vec(4, np.float64)
spatial_matrix, spatial_matrixd = _Mat(6, 6, np.float32), _Mat(6, 6, np.float64)
spatial_vector, spatial_vectord = _Vec(6, np.float32), _Vec(6, np.float64)


class _Types:
    @staticmethod
    def matrix(shape, dtype):
        return _Mat(shape[0], shape[1], dtype)

    @staticmethod
    def vector(length, dtype):
        return _Vec(length, dtype)


types_ = _Types()


def array(*args, dtype=None, **kw):
    """Annotation placeholder, or a numpy array when data is given."""
    if args and not isinstance(args[0], type):
        return np.array(args[0], dtype=dtype)
    return ("array", dtype)


def array2d(*args, dtype=None, **kw):
    return ("array2d", dtype)


# --------------------------------------------------------------- builtins
def _is_vec(a):
    return isinstance(a, np.ndarray)


def dot(a, b):
    if a.ndim == 2:  # matrix ddot not used on this path
        raise NotImplementedError
    acc = a[0] * b[0]
    for i in range(1, a.shape[0]):
        acc = acc + a[i] * b[i]
    return acc


def cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]],
                    dtype=np.result_type(a, b))


def length(a):
    d = dot(a, a)
    return type(d)(math.sqrt(d))


def length_sq(a):
    return dot(a, a)


def normalize(a):
    return a / length(a)


def sqrt(x):
    return type(x)(math.sqrt(x)) if isinstance(x, np.floating) else math.sqrt(x)


def abs(x):  # noqa: A001
    return np.abs(x)


def min(a, b):  # noqa: A001
    if _is_vec(a):
        return np.where(a < b, a, b).astype(a.dtype)
    return a if a < b else b


def max(a, b):  # noqa: A001
    if _is_vec(a):
        return np.where(a > b, a, b).astype(a.dtype)
    return a if a > b else b


def clamp(x, lo, hi):
    return lo if x < lo else (hi if x > hi else x)


def lerp(a, b, t):
    return a * (type(t)(1.0) - t) + b * t


def outer(a, b):
    return np.outer(a, b).astype(np.result_type(a, b))


def matrix_from_cols(*cols):
    return np.stack(cols, axis=1)


def ddot(a, b):
    """Frobenius product, summed row by row in the matrix's scalar type."""
    acc = a[0, 0] * b[0, 0]
    for i in range(a.shape[0]):
        for j in range(a.shape[1]):
            if i or j:
                acc = acc + a[i, j] * b[i, j]
    return acc


def trace(m):
    acc = m[0, 0]
    for i in range(1, m.shape[0]):
        acc = acc + m[i, i]
    return acc


def determinant(m):
    """3x3 cofactor expansion along the first row, in the scalar type."""
    return (m[0, 0] * (m[1, 1] * m[2, 2] - m[1, 2] * m[2, 1])
            - m[0, 1] * (m[1, 0] * m[2, 2] - m[1, 2] * m[2, 0])
            + m[0, 2] * (m[1, 0] * m[2, 1] - m[1, 1] * m[2, 0]))


def inverse(m):
    """3x3 adjugate over the determinant, in the scalar type."""
    d = determinant(m)
    adj = np.empty_like(m)
    for i in range(3):
        for j in range(3):
            r = [k for k in range(3) if k != j]
            c = [k for k in range(3) if k != i]
            minor = m[r[0], c[0]] * m[r[1], c[1]] - m[r[0], c[1]] * m[r[1], c[0]]
            adj[i, j] = minor if (i + j) % 2 == 0 else -minor
    return adj / d


def identity(n=3, dtype=np.float32):
    return np.eye(n, dtype=dtype)


def log(x):
    return type(x)(math.log(x)) if isinstance(x, np.floating) else math.log(x)


def transpose(m):
    return m.T.copy()


def _wrap32(x):
    x = int(x) & 0xFFFFFFFF
    return x - (1 << 32) if x >= (1 << 31) else x


def bit_xor(a, b):
    """int32 semantics (products wrap, as in the compiled kernel)."""
    return _wrap32(_wrap32(a) ^ _wrap32(b))


def atomic_add(arr, idx, val):
    old = arr[idx].copy() if isinstance(arr[idx], np.ndarray) else arr[idx]
    arr[idx] = arr[idx] + val
    return old


def atomic_min(arr, idx, val):
    old = arr[idx]
    if val < arr[idx]:
        arr[idx] = val
    return old


def closest_point_edge_edge(p1, q1, p2, q2, epsilon):
    """Ericson RTCD 5.1.9 in float32; returns vec3(s, t, dist)."""
    f32 = np.float32
    eps = f32(epsilon)
    d1, d2, r = q1 - p1, q2 - p2, p1 - p2
    a, e, f = dot(d1, d1), dot(d2, d2), dot(d2, r)
    s = t = f32(0.0)
    if a <= eps and e <= eps:
        pass
    elif a <= eps:
        t = clamp(f / e, f32(0), f32(1))
    else:
        c = dot(d1, r)
        if e <= eps:
            s = clamp(-c / a, f32(0), f32(1))
        else:
            b = dot(d1, d2)
            denom = a * e - b * b
            s = clamp((b * f - c * e) / denom, f32(0), f32(1)) if denom != 0 else f32(0)
            t = (b * s + f) / e
            if t < 0:
                t = f32(0)
                s = clamp(-c / a, f32(0), f32(1))
            elif t > 1:
                t = f32(1)
                s = clamp((b - c) / a, f32(0), f32(1))
    c1, c2 = p1 + d1 * s, p2 + d2 * t
    return np.array([s, t, length(c1 - c2)], dtype=np.float32)


# ---------------------------------------------------------- BVH stand-ins
class BoxSet:
    """A 'BVH id': boxes (n, 3) float32 lower/upper."""

    def __init__(self, lower, upper):
        self.lower = np.asarray(lower, np.float32)
        self.upper = np.asarray(upper, np.float32)


def bvh_query_aabb(bvh: BoxSet, low, high):
    lo, hi = np.asarray(low, np.float32), np.asarray(high, np.float32)
    ok = np.all(bvh.lower <= hi, axis=1) & np.all(lo <= bvh.upper, axis=1)
    return iter(np.flatnonzero(ok).tolist())


mesh_query_aabb = bvh_query_aabb
