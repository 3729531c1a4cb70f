"""CPU restatement of the mixed FEM + affine-body Newton system (test
infrastructure only; the product never imports this module).

The reference has no solver that mixes tets and affine bodies; its two
solvers supply the terms: the tet part of time_integrator_base.py:403-438
(oracle/newton.py, pyoracle.tet), the affine part of
affine_body_dynamics.py:88-217 (oracle/abd.py) and the contact terms of
dynamic_contacts.py:249-308 (pyoracle.dcd_* / narrow).  Here they are
combined over one unknown vector q = [FEM vertex positions; p, a0, a1, a2
per body]: the contact force and Hessian of the vertices are pulled back
with the explicit Jacobian J (x = J q), and a pin (pendulum rod) adds
0.5 h^2 k |x_pin - target|^2 per pinned body.  Everything is in double with
scipy sparse matrices.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from . import abd as oabd
from . import newton as on
from . import pyoracle as po


@dataclass
class Mixed:
    n_fem: int
    body: np.ndarray         # (V - n_fem,) body of each affine vertex
    fixed: np.ndarray        # (nb,) 1 = fixed body
    rest: np.ndarray         # (V, 3) soup xcs: FEM rest, then body-local rest
    fem_mass: np.ndarray     # (n_fem,)
    M: np.ndarray            # (nb, 4, 4) mass moments
    volume: np.ndarray       # (nb,)
    stiffness: np.ndarray    # (nb,)
    pin_rest: np.ndarray     # (nb, 3) body-local pin points
    pin_target: np.ndarray   # (nb, 3)
    pin_k: np.ndarray        # (nb,)

    @property
    def nb(self):
        return len(self.volume)

    @property
    def nq(self):
        return self.n_fem + 4 * self.nb


def jacobian(m: Mixed) -> sp.csr_matrix:
    """d x / d q (3V x 3 nq): I for FEM vertices, [I, r0 I, r1 I, r2 I] for
    vertices of free bodies, nothing for fixed bodies."""
    V = len(m.rest)
    rows, cols, vals = [], [], []
    for v in range(V):
        if v < m.n_fem:
            dofs, w = [v], [1.0]
        else:
            b = m.body[v - m.n_fem]
            if m.fixed[b]:
                continue
            dofs = [m.n_fem + 4 * b + k for k in range(4)]
            w = [1.0, *m.rest[v]]
        for d, wk in zip(dofs, w):
            for c in range(3):
                rows.append(3 * v + c)
                cols.append(3 * d + c)
                vals.append(wk)
    return sp.csr_matrix((vals, (rows, cols)), shape=(3 * V, 3 * m.nq))


def vertex_positions(m: Mixed, q: np.ndarray) -> np.ndarray:
    return (jacobian(m) @ np.asarray(q, np.float64).reshape(-1)).reshape(-1, 3) + _fixed_positions(m, q)


def _fixed_positions(m: Mixed, q):
    """Vertices of fixed bodies keep x = p + A r of their (unchanging) q."""
    q = np.asarray(q, np.float64).reshape(-1, 3)
    out = np.zeros((len(m.rest), 3))
    for v in range(m.n_fem, len(m.rest)):
        b = m.body[v - m.n_fem]
        if m.fixed[b]:
            Q = q[m.n_fem + 4 * b:m.n_fem + 4 * b + 4]
            out[v] = Q[0] + m.rest[v] @ Q[1:]
    return out


def _pins(m: Mixed, q, h2):
    """Pin energy, gradient (nq, 3) and 3nq x 3nq Hessian."""
    q = np.asarray(q, np.float64).reshape(-1, 3)
    e = 0.0
    g = np.zeros_like(q)
    rows, cols, vals = [], [], []
    for b in range(m.nb):
        k = m.pin_k[b]
        if k == 0 or m.fixed[b]:
            continue
        o = m.n_fem + 4 * b
        w = np.concatenate(([1.0], m.pin_rest[b]))
        x = w @ q[o:o + 4]
        r = x - m.pin_target[b]
        e += 0.5 * h2 * k * float(r @ r)
        for i in range(4):
            g[o + i] += h2 * k * w[i] * r
            for j in range(4):
                for c in range(3):
                    rows.append(3 * (o + i) + c)
                    cols.append(3 * (o + j) + c)
                    vals.append(h2 * k * w[i] * w[j])
    H = sp.csr_matrix((vals, (rows, cols)), shape=(3 * m.nq, 3 * m.nq))
    return e, g, H


def system(p: on.Problem, m: Mixed, q, xt_f, qt_a, x=None):
    """Gradient (nq, 3) and Newton matrix (scipy CSR, 3 nq square) at q;
    ``x`` overrides the vertex positions the contact and tet terms read
    (the GPU's rounded J q).  Returns (g, A, n_ee, n_pt)."""
    h2 = p.h * p.h
    q = np.asarray(q, np.float64).reshape(-1, 3)
    Vf, nb = m.n_fem, m.nb
    V = len(m.rest)
    xv = vertex_positions(m, q) if x is None else np.asarray(x)
    xs = np.asarray(xv, dtype=p.dtype).astype(np.float64)
    # vertex-space force and Hessian: tets and contact
    force, blocks, _ = po.tet(p.material, xs, p.xcs, p.tets, p.mu, p.lam)
    R, C, B = [], [], []
    T = p.tets.reshape(-1, 4)
    if len(T):
        R.append(np.repeat(T, 4, axis=1).reshape(-1))
        C.append(np.tile(T, (1, 4)).reshape(-1))
        B.append(blocks.reshape(-1, 3, 3))
    ee, pt, l0 = on._contacts(p, xv)
    for idx, F, H, _ in on._narrow(p, xv, ee, pt, l0):
        for k in range(4):
            np.add.at(force, idx[:, k], F[:, 3 * k:3 * k + 3])
        if len(idx):
            R.append(np.repeat(idx, 4, axis=1).reshape(-1))
            C.append(np.tile(idx, (1, 4)).reshape(-1))
            B.append(H.reshape(-1, 4, 3, 4, 3).transpose(0, 1, 3, 2, 4).reshape(-1, 3, 3))
    if R:
        R, C, B = np.concatenate(R), np.concatenate(C), np.concatenate(B)
        r = (3 * R[:, None, None] + np.arange(3)[None, :, None]).repeat(3, axis=2)
        c = (3 * C[:, None, None] + np.arange(3)[None, None, :]).repeat(3, axis=1)
        Hv = sp.csr_matrix((B.ravel(), (r.ravel(), c.ravel())), shape=(3 * V, 3 * V))
    else:
        Hv = sp.csr_matrix((3 * V, 3 * V))
    J = jacobian(m)
    A = h2 * (J.T @ Hv @ J)
    g = (-h2 * (J.T @ force.reshape(-1))).reshape(-1, 3)
    # FEM inertia
    d = np.arange(3 * Vf)
    A = A + sp.csr_matrix((np.repeat(m.fem_mass, 3), (d, d)), shape=A.shape)
    g[:Vf] += m.fem_mass[:, None] * (q[:Vf] - xt_f)
    # bodies
    if nb:
        blk, grad = oabd.body_system(q[Vf:].reshape(-1, 4, 3), np.asarray(qt_a).reshape(-1, 4, 3), m.M, m.volume,
                                     m.stiffness, m.fixed, h2)
        rows, cols, vals = [], [], []
        for b in range(nb):
            full = blk[b].transpose(0, 2, 1, 3).reshape(12, 12)
            base = 3 * (Vf + 4 * b)
            ii, jj = np.meshgrid(np.arange(12), np.arange(12), indexing="ij")
            rows.append((base + ii).ravel())
            cols.append((base + jj).ravel())
            vals.append(full.ravel())
        A = A + sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=A.shape)
        g[Vf:] += grad.reshape(-1, 3)
        _, gp, Hp = _pins(m, q, h2)
        A = A + Hp
        g += gp
    return g, A.tocsr(), len(ee), len(pt)


def energy(p: on.Problem, m: Mixed, q, xt_f, qt_a, x=None) -> float:
    """h^2 Psi + FEM inertia + body inertia + h^2 orthogonality + pins +
    h^2 barrier at q."""
    h2 = p.h * p.h
    q = np.asarray(q, np.float64).reshape(-1, 3)
    Vf = m.n_fem
    xv = vertex_positions(m, q) if x is None else np.asarray(x)
    xs = np.asarray(xv, dtype=p.dtype).astype(np.float64)
    _, _, psi = po.tet(p.material, xs, p.xcs, p.tets, p.mu, p.lam)
    d = q[:Vf] - xt_f
    inertia = 0.5 * float((m.fem_mass[:, None] * d * d).sum())
    bi = bo = pe = 0.0
    if m.nb:
        bi, bo = oabd.body_energy(q[Vf:].reshape(-1, 4, 3), np.asarray(qt_a).reshape(-1, 4, 3), m.M, m.volume,
                                  m.stiffness, m.fixed, h2)
        pe, _, _ = _pins(m, q, h2)
    ee, pt, l0 = on._contacts(p, xv)
    barrier = sum(float(E.sum()) for _, _, _, E in on._narrow(p, xv, ee, pt, l0))
    return h2 * psi + inertia + bi + bo + pe + h2 * barrier


def from_scene(scene, E: float = 1e5, nu: float = 0.4, rho: float = 1000.0, density: float = 1000.0,
               affine_stiffness: float = 1e5, h: float = 1e-2, material: int = 1, fp64: bool = True):
    """(Problem, Mixed, q) of a MixedScene at rest, set up as
    ipc_warp_b200.mixed.MixedSolver does (FEM vertices first, then the
    bodies' surfaces; body-local rest positions about the volume
    centroids)."""
    fem = scene.fem
    Vf = fem.n_verts
    nb = len(scene.bodies)
    bv, bf, bb = [], [], []
    off = Vf
    for b, (v, f) in enumerate(scene.bodies):
        bv.append(np.asarray(v, np.float64))
        bf.append(np.asarray(f, np.int64).reshape(-1, 3) + off)
        bb.append(np.full(len(v), b, np.int32))
        off += len(v)
    world = np.concatenate(bv)
    faces = np.concatenate(bf)
    body = np.concatenate(bb)
    fixed = np.zeros(nb, np.int32)
    fixed[list(scene.fixed_bodies)] = 1
    centers, volumes, weights = oabd.mass_properties(world, faces - Vf, body)
    local = world - centers[body]
    xcs = np.concatenate([fem.xcs, local])
    e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
    edges = np.concatenate([fem.edges.reshape(-1, 2), np.unique(np.sort(e, axis=1), axis=0)])
    tris = np.concatenate([fem.triangles.reshape(-1, 3), faces])
    soup_body = np.concatenate([fem.body, body + int(fem.body.max()) + 1])
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    V = len(xcs)
    p = on.Problem(xcs=xcs, tets=fem.tets, edges=edges, triangles=tris, body=soup_body, mass=np.zeros(V),
                   fixed=np.zeros(V, bool), x_target=np.zeros((V, 3)), material=material, mu=mu, lam=lam,
                   dhat=scene.dhat, kappa=scene.kappa, h=h, k_att=0.0, gravity=np.zeros(3), fp64=fp64,
                   exclude_same_body=True)
    pr, pt, pk = np.zeros((nb, 3)), np.zeros((nb, 3)), np.zeros(nb)
    for b, (point, target, k) in (scene.pins or {}).items():
        pr[b] = np.asarray(point) - centers[b]
        pt[b] = target
        pk[b] = k
    m = Mixed(n_fem=Vf, body=body, fixed=fixed, rest=xcs, fem_mass=on.lumped_mass(fem.xcs, fem.tets, rho),
              M=oabd.mass_moments(local, body, weights, volumes, density), volume=volumes,
              stiffness=np.full(nb, float(affine_stiffness)), pin_rest=pr, pin_target=pt, pin_k=pk)
    q = np.zeros((m.nq, 3))
    q[:Vf] = fem.x
    qa = np.zeros((nb, 4, 3))
    qa[:, 0] = centers
    qa[:, 1:] = np.eye(3)
    q[Vf:] = qa.reshape(-1, 3)
    return p, m, q
