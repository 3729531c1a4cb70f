"""ctypes binding of the CPU oracle (oracle/oracle.cpp).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "liboracle.so")
SOURCES = [os.path.join(_HERE, "oracle.cpp")]


def build(force: bool = False) -> str:
    """Compile the oracle with g++ (-O3 -fopenmp -ffp-contract=off)."""
    os.makedirs(os.path.dirname(LIB_PATH), exist_ok=True)
    newest = max(os.path.getmtime(s) for s in SOURCES)
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-Wall", "-Wno-unused-function", *SOURCES, "-o", LIB_PATH]
    subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def closest_point_triangle(p, a, b, c):
    p, a, b, c = (_f32(v).reshape(-1, 3) for v in (p, a, b, c))
    n = p.shape[0]
    uvd = np.zeros((n, 3), np.float32)
    ty = np.zeros(n, np.int32)
    lib().ora_closest_point_triangle(n, _p(p), _p(a), _p(b), _p(c), _p(uvd), _p(ty))
    return uvd, ty


def closest_point_edge_edge(p1, q1, p2, q2, eps=1e-6):
    p1, q1, p2, q2 = (_f32(v).reshape(-1, 3) for v in (p1, q1, p2, q2))
    n = p1.shape[0]
    out = np.zeros((n, 3), np.float32)
    lib().ora_closest_point_edge_edge(n, _p(p1), _p(q1), _p(p2), _p(q2), ctypes.c_float(eps), _p(out))
    return out


def _dcd(fn, nv, x, prims, body, th, exclude, cap):
    x = _f32(x).reshape(-1)
    prims = _i32(prims).reshape(-1)
    body = _i32(body)
    out = np.zeros((cap, 6), np.int32)
    n = fn(nv, _p(x), prims.size // (2 if fn is lib().ora_dcd_ee else 3), _p(prims), _p(body),
           ctypes.c_float(th), int(exclude), _p(out), cap)
    if n > cap:
        return _dcd(fn, nv, x, prims, body, th, exclude, n)
    return out[:n]


def dcd_ee(x, edges, body, th, exclude_same_body=False, cap=1 << 16):
    """EE candidates [(a1,a2,b1,b2,i,j)] (contact.py:199-228), unsorted."""
    x = np.asarray(x)
    return _dcd(lib().ora_dcd_ee, x.shape[0], x, edges, body, th, exclude_same_body, cap)


def dcd_pt(x, triangles, body, th, exclude_same_body=False, cap=1 << 16):
    """PT candidates [(p, t1, t0, t2, p, tri)] (contact.py:304-336), unsorted."""
    x = np.asarray(x)
    return _dcd(lib().ora_dcd_pt, x.shape[0], x, triangles, body, th, exclude_same_body, cap)


def narrow(kind: str, idx, l0, x, xcs, kappa, fp64=False, mode=0):
    """Per-pair force (n,12), Hessian (n,12,12), energy (n,), active flags."""
    dt = np.float64 if fp64 else np.float32
    idx = _i32(idx).reshape(-1, 4)
    n = idx.shape[0]
    l0 = np.ascontiguousarray(l0, dtype=dt)
    x = np.ascontiguousarray(x, dtype=dt).reshape(-1)
    xcs = np.ascontiguousarray(xcs if xcs is not None else x, dtype=dt).reshape(-1)
    force = np.zeros((n, 12))
    hess = np.zeros((n, 12, 12))
    energy = np.zeros(n)
    active = np.zeros(n, np.int32)
    lib().ora_narrow(int(kind == "ee"), int(fp64), int(mode), n, _p(idx), _p(l0), _p(x), _p(xcs),
                     ctypes.c_double(kappa), _p(force), _p(hess), _p(energy), _p(active))
    return force, hess, energy, active


def feature_dh(kind: int, pts, mode=0):
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(12)
    g = np.zeros(12)
    h = np.zeros((12, 12))
    lib().ora_feature_dh(int(kind), int(mode), _p(pts), _p(g), _p(h))
    return g, h


def barrier(x, xh, kappa):
    x = np.ascontiguousarray(x, dtype=np.float64)
    xh = np.ascontiguousarray(np.broadcast_to(xh, x.shape), dtype=np.float64)
    out = np.zeros((x.size, 3))
    lib().ora_barrier(x.size, _p(x), _p(xh), ctypes.c_double(kappa), _p(out))
    return out


def cubic_roots(coef, x0, x1):
    coef = np.ascontiguousarray(coef, dtype=np.float64).reshape(-1, 4)
    n = coef.shape[0]
    roots = np.zeros((n, 3))
    nr = np.zeros(n, np.int32)
    st = lib().ora_cubic_roots(n, _p(coef), ctypes.c_double(x0), ctypes.c_double(x1), _p(roots), _p(nr))
    return nr, roots, st


def collision_time(kind: str, p_t0, p_t1):
    a = np.ascontiguousarray(p_t0, dtype=np.float64).reshape(-1, 12)
    b = np.ascontiguousarray(p_t1, dtype=np.float64).reshape(-1, 12)
    t = np.zeros(a.shape[0])
    lib().ora_collision_time(int(kind == "ee"), a.shape[0], _p(a), _p(b), _p(t))
    return t


def scene_toi(x0, x1, edges, triangles, body, exclude_same_body=False, fp64=False):
    """Minimum TOI (< 1) over all swept-box-overlapping EE and PT pairs, or 1."""
    dt = np.float64 if fp64 else np.float32
    x0 = np.ascontiguousarray(x0, dtype=dt).reshape(-1, 3)
    x1 = np.ascontiguousarray(x1, dtype=dt).reshape(-1, 3)
    edges, triangles, body = _i32(edges).reshape(-1), _i32(triangles).reshape(-1), _i32(body)
    st = np.zeros(1, np.int32)
    f = lib().ora_scene_toi
    f.restype = ctypes.c_double
    t = f(int(fp64), x0.shape[0], _p(x0), _p(x1), edges.size // 2, _p(edges), triangles.size // 3, _p(triangles),
          _p(body), int(exclude_same_body), _p(st))
    return float(t), int(st[0])


def tet(material: int, x, xcs, tets, mu, lam):
    """Elastic force (V,3), per-tet 16 blocks (n,16,3,3) and energy (double)."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
    xcs = np.ascontiguousarray(xcs, dtype=np.float64).reshape(-1, 3)
    tets = _i32(tets).reshape(-1, 4)
    force = np.zeros_like(x)
    blocks = np.zeros((tets.shape[0], 16, 3, 3))
    f = lib().ora_tet
    f.restype = ctypes.c_double
    e = f(int(material), x.shape[0], _p(x), _p(xcs), tets.shape[0], _p(tets), ctypes.c_double(mu),
          ctypes.c_double(lam), _p(force), _p(blocks))
    return force, blocks, float(e)


def contact_bsr(nv, idx, hess):
    """Contact BSR (offsets, columns, values (nnz, 3, 3)) of records idx (n, 4)
    with 12x12 Hessians hess (n, 12, 12), dynamic_contacts.py:281-297."""
    idx = _i32(idx).reshape(-1, 4)
    hess = np.ascontiguousarray(hess, dtype=np.float64).reshape(-1, 12, 12)
    n = idx.shape[0]
    offsets = np.zeros(nv + 1, np.int32)
    cap = 16 * n
    cols = np.zeros(max(cap, 1), np.int32)
    vals = np.zeros((max(cap, 1), 3, 3))
    nnz = lib().ora_contact_bsr(int(nv), n, _p(idx), _p(hess), _p(offsets), _p(cols), _p(vals), cap)
    return offsets, cols[:nnz], vals[:nnz]


def edge_triangle_crossings(x, edges, triangles, cap=1 << 16):
    """(count, pairs (m, 2) sorted) of surface edges strictly crossing
    surface triangles without a shared vertex (the intersection check)."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
    edges, triangles = _i32(edges).reshape(-1), _i32(triangles).reshape(-1)
    out = np.zeros((max(cap, 1), 2), np.int32)
    n = lib().ora_edge_triangle_crossings(x.size // 3, _p(x), edges.size // 2, _p(edges), triangles.size // 3,
                                          _p(triangles), _p(out), cap)
    return n, out[:min(n, cap)]
