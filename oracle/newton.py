"""CPU restatement of one implicit-Euler Newton step with IPC contact
(test infrastructure only; the product never imports this module).

Follows time_integrator_base.py:375-546 (``RodBCBase.step``, ``compute_A``,
``compute_rhs``, ``line_search``) with the contact terms of
dynamic_contacts.py:249-308: the elastic term is ``pyoracle.tet``, contact
candidates ``pyoracle.dcd_ee/dcd_pt``, the barrier ``pyoracle.narrow`` and the
line-search bound ``pyoracle.scene_toi``; the linear system is solved
directly (scipy sparse LU) in double.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import pyoracle as po


@dataclass
class Problem:
    xcs: np.ndarray          # (V, 3) rest positions
    tets: np.ndarray         # (T, 4)
    edges: np.ndarray        # (E, 2)
    triangles: np.ndarray    # (F, 3)
    body: np.ndarray         # (V,)
    mass: np.ndarray         # (V,) lumped
    fixed: np.ndarray        # (V,) bool
    x_target: np.ndarray     # (V, 3)
    material: int
    mu: float
    lam: float
    dhat: float
    kappa: float
    h: float
    k_att: float
    gravity: np.ndarray      # (3,)
    fp64: bool = False
    exclude_same_body: bool = False

    @property
    def dtype(self):
        return np.float64 if self.fp64 else np.float32


def lumped_mass(xcs, tets, rho):
    X = xcs[tets]
    Dm = np.stack([X[:, i] - X[:, 3] for i in range(3)], axis=2)
    w = np.abs(np.linalg.det(Dm)) / 6.0
    m = np.zeros(len(xcs))
    np.add.at(m, tets.reshape(-1), np.repeat(rho * w / 4.0, 4))
    m[m == 0] = rho * (w.mean() if len(w) else 1.0) / 4.0
    return m


def _contacts(p: Problem, x):
    """EE and PT records at x (float32 queries, as the GPU pipeline)."""
    x32 = np.asarray(x, dtype=np.float32)
    th = np.float32(0.5 * p.dhat)
    ee = po.dcd_ee(x32, p.edges, p.body, th, p.exclude_same_body)
    pt = po.dcd_pt(x32, p.triangles, p.body, th, p.exclude_same_body) if len(p.triangles) else np.zeros((0, 6), np.int32)
    l0 = p.dtype(th) * p.dtype(2.0)
    return ee, pt, l0


def _narrow(p: Problem, x, ee, pt, l0):
    xs = np.asarray(x, dtype=p.dtype)
    out = []
    for kind, rec in (("ee", ee), ("pt", pt)):
        if len(rec) == 0:
            out.append((rec[:, :4], np.zeros((0, 12)), np.zeros((0, 12, 12)), np.zeros(0)))
            continue
        F, H, E, _ = po.narrow(kind, rec[:, :4], np.full(len(rec), l0, p.dtype), xs,
                               p.xcs if kind == "ee" else None, p.kappa, fp64=p.fp64, mode=1)
        out.append((rec[:, :4], F, H, E))
    return out


def x_tilde(p: Problem, x0, xdot):
    return x0 + p.h * xdot + p.h * p.h * p.gravity


def energy(p: Problem, x, xt) -> float:
    """h^2 Psi + 1/2 |x - x~|_M^2 + h^2 B + 1/2 h^2 k_att |x - x_target|^2_fixed."""
    h2 = p.h * p.h
    xs = np.asarray(x, dtype=p.dtype).astype(np.float64)
    _, _, psi = po.tet(p.material, xs, p.xcs, p.tets, p.mu, p.lam)
    d = xs - xt
    inertia = 0.5 * float((p.mass[:, None] * d * d).sum())
    ee, pt, l0 = _contacts(p, x)
    barrier = sum(float(E.sum()) for _, _, _, E in _narrow(p, x, ee, pt, l0))
    r = (xs - p.x_target)[p.fixed]
    att = 0.5 * p.k_att * h2 * float((r * r).sum())
    return h2 * psi + inertia + h2 * barrier + att


def gradient_hessian(p: Problem, x, xt):
    """Gradient (V, 3) and the Newton matrix (scipy CSR, 3V x 3V)."""
    h2 = p.h * p.h
    V = len(p.xcs)
    xs = np.asarray(x, dtype=p.dtype).astype(np.float64)
    force, blocks, _ = po.tet(p.material, xs, p.xcs, p.tets, p.mu, p.lam)
    rows, cols, vals = [], [], []
    T = p.tets.reshape(-1, 4)
    rows.append(np.repeat(T, 4, axis=1).reshape(-1))
    cols.append(np.tile(T, (1, 4)).reshape(-1))
    vals.append(h2 * blocks.reshape(-1, 3, 3))
    ee, pt, l0 = _contacts(p, x)
    for idx, F, H, _ in _narrow(p, x, ee, pt, l0):
        for k in range(4):
            np.add.at(force, idx[:, k], F[:, 3 * k:3 * k + 3])
        Hb = H.reshape(-1, 4, 3, 4, 3).transpose(0, 1, 3, 2, 4).reshape(-1, 3, 3)
        rows.append(np.repeat(idx, 4, axis=1).reshape(-1))
        cols.append(np.tile(idx, (1, 4)).reshape(-1))
        vals.append(h2 * Hb)
    diag = p.mass[:, None, None] * np.eye(3) + (h2 * p.k_att) * p.fixed[:, None, None] * np.eye(3)
    rows.append(np.arange(V))
    cols.append(np.arange(V))
    vals.append(diag)
    R, C, Vb = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    r = (3 * R[:, None, None] + np.arange(3)[None, :, None]).repeat(3, axis=2)
    c = (3 * C[:, None, None] + np.arange(3)[None, None, :]).repeat(3, axis=1)
    A = sp.coo_matrix((Vb.ravel(), (r.ravel(), c.ravel())), shape=(3 * V, 3 * V)).tocsr()
    g = -h2 * force + p.mass[:, None] * (xs - xt) + (h2 * p.k_att) * p.fixed[:, None] * (xs - p.x_target)
    return g, A


def line_search(p: Problem, x, dx, xt):
    """time_integrator_base.py:514-546 with the CCD bound of
    contact.py:539-585 (0.9 toi when toi < 1)."""
    E0 = energy(p, x, xt)
    toi, _ = po.scene_toi(np.asarray(x, p.dtype), np.asarray(x - dx, p.dtype), p.edges, p.triangles, p.body,
                          p.exclude_same_body, fp64=p.fp64)
    ub = 0.9 * toi if toi < 1.0 else 1.0
    alpha = ub
    eps = float(np.finfo(p.dtype).eps)
    for _ in range(64):
        xn = (x - alpha * dx).astype(p.dtype)
        E1 = energy(p, xn, xt)
        if math.isfinite(E1) and E1 < E0:
            return xn, alpha, E0, E1
        alpha *= 0.5
        if alpha <= eps * max(1.0, ub):
            break
    return x, 0.0, E0, E0


def step(p: Problem, x0, xdot, vel_tol=5e-2, max_newton=100):
    """One time step; returns (x, xdot, per-iteration [(alpha, max|dx|)])."""
    xt = x_tilde(p, np.asarray(x0, np.float64), np.asarray(xdot, np.float64))
    x = np.asarray(x0, dtype=p.dtype).copy()
    log = []
    for _ in range(max_newton):
        g, A = gradient_hessian(p, x, xt)
        dx = spla.spsolve(A.tocsc(), g.reshape(-1)).reshape(-1, 3)
        x, alpha, _, _ = line_search(p, x, dx, xt)
        norm = float(np.abs(dx).max()) if alpha > 0 else 0.0
        log.append((alpha, norm))
        if alpha == 0.0 or norm <= vel_tol * p.h:
            break
    xd = (x.astype(np.float64) - np.asarray(x0, np.float64)) / p.h
    return x, xd, log
