"""CPU restatement of the affine-body (ABD) terms (test infrastructure only;
the product never imports this module).

Follows affine_body_dynamics.py: the vertex map x = p + r0 a0 + r1 a1 + r2 a2
(_sync_affine_vertices 42-48, _affine_vertex_direction 51-57), the predictor
(_prepare_tilde 66-79), the velocity update (_update_affine_velocity 82-86),
the per-body 4x4 system of inertia plus orthogonality potential
(_assemble_body_system 88-141), the vertex->affine reductions of the contact
force and Hessian (_reduce_contact_force 144-157, _reduce_contact_hessian
166-190), the energies (_body_energy 193-217), and the host-side mass
properties (_mass_properties 318-342, _build_mass_blocks 344-358).

q is (nb, 4, 3): per body p, a0, a1, a2 (the columns of A).  Mass blocks are
the scalar moments M (nb, 4, 4); the reference stores M_ij * I as mat33.

Parity pin: the reference's Warp kernels cannot run here (no Warp), so this
restatement is pinned by identities instead: the gradient and Hessian are
the derivatives of the energy (finite differences), the reductions equal
J^T f and J^T H J with the explicit affine Jacobian, and the mass moments of
a closed surface equal its analytic volume and centroid.
"""
from __future__ import annotations

import numpy as np

from . import newton as on


def mass_properties(vertices, faces, body):
    """affine_body_dynamics.py:318-342: volume centroid, |volume| and the
    per-vertex area weights (a third of every incident triangle's area)."""
    vertices = np.asarray(vertices, np.float64)
    faces = np.asarray(faces).reshape(-1, 3)
    nb = int(body.max()) + 1
    centers = np.zeros((nb, 3))
    volumes = np.zeros(nb)
    weights = np.zeros(len(vertices))
    for b in range(nb):
        fb = faces[body[faces[:, 0]] == b]
        if len(fb) == 0:
            centers[b] = vertices[body == b].mean(axis=0)
            volumes[b] = 1.0
            weights[body == b] = 1.0
            continue
        a, c, d = vertices[fb[:, 0]], vertices[fb[:, 1]], vertices[fb[:, 2]]
        signed = np.einsum("ij,ij->i", a, np.cross(c, d)) / 6.0
        total = signed.sum()
        if abs(total) > 1e-12:
            centers[b] = (signed[:, None] * (a + c + d) / 4.0).sum(axis=0) / total
            volumes[b] = abs(total)
        else:
            centers[b] = vertices[body == b].mean(axis=0)
            volumes[b] = max(float(np.prod(np.ptp(vertices[body == b], axis=0))), 1e-12)
        area = 0.5 * np.linalg.norm(np.cross(c - a, d - a), axis=1)
        for k in range(3):
            np.add.at(weights, fb[:, k], area / 3.0)
    return centers, volumes, weights


def mass_moments(local, body, weights, volumes, density):
    """affine_body_dynamics.py:344-358: M_b = sum_v w_v [1, r_v][1, r_v]^T with
    the weights scaled to the body mass density * volume."""
    nb = len(volumes)
    M = np.zeros((nb, 4, 4))
    for b in range(nb):
        ids = np.flatnonzero(body == b)
        w = weights[ids]
        m = density * float(volumes[b])
        w = np.full(len(ids), m / len(ids)) if w.sum() == 0 else w / w.sum() * m
        C = np.column_stack((np.ones(len(ids)), local[ids]))
        M[b] = C.T @ (w[:, None] * C)
    return M


def affine_map(q, rest, body):
    """x_v = q[b,0] + sum_k r_v[k] q[b,k+1]."""
    q = np.asarray(q).reshape(-1, 4, 3)
    Q = q[body]
    return Q[:, 0] + np.einsum("vk,vkj->vj", rest, Q[:, 1:])


def prepare_tilde(q0, qdot, h, gravity, omega, enabled):
    """affine_body_dynamics.py:66-79."""
    q0 = np.asarray(q0).reshape(-1, 4, 3)
    qdot = np.asarray(qdot).reshape(-1, 4, 3)
    qt = q0 + h * qdot
    qt[:, 0] += h * h * np.asarray(gravity)
    for b in np.flatnonzero(enabled):
        qt[b, 1:] = q0[b, 1:] + h * np.cross(omega[b], q0[b, 1:])
    return qt


def update_velocity(q, q0, h):
    return (np.asarray(q) - np.asarray(q0)) / h, np.array(q, copy=True)


def _ortho(a):
    """Gradient/4 and Hessian/4 (block (i, j) of the 3 columns) of
    sum_i (|a_i|^2 - 1)^2 + 2 sum_{i<j} (a_i . a_j)^2."""
    g = np.zeros((3, 3))
    H = np.zeros((3, 3, 3, 3))
    I = np.eye(3)
    for i in range(3):
        g[i] = (a[i] @ a[i] - 1.0) * a[i] + sum((a[i] @ a[k]) * a[k] for k in range(3) if k != i)
        for j in range(3):
            if i == j:
                H[i, j] = (a[i] @ a[i] - 1.0) * I + 2.0 * np.outer(a[i], a[i]) + sum(
                    np.outer(a[k], a[k]) for k in range(3) if k != i)
            else:
                H[i, j] = (a[i] @ a[j]) * I + np.outer(a[j], a[i])
    return g, H


def body_system(q, qt, M, volume, stiffness, fixed, h2):
    """affine_body_dynamics.py:88-141: the 16 blocks (nb, 4, 4, 3, 3) and the
    gradient (nb, 4, 3) of inertia + orthogonality potential."""
    q = np.asarray(q, np.float64).reshape(-1, 4, 3)
    qt = np.asarray(qt, np.float64).reshape(-1, 4, 3)
    nb = len(q)
    blocks = np.zeros((nb, 4, 4, 3, 3))
    grad = np.zeros((nb, 4, 3))
    I = np.eye(3)
    for b in range(nb):
        if fixed[b]:
            for i in range(4):
                blocks[b, i, i] = I
            continue
        for i in range(4):
            for j in range(4):
                blocks[b, i, j] = M[b, i, j] * I
        grad[b] = M[b] @ (q[b] - qt[b])
        s = 4.0 * stiffness[b] * volume[b] * h2
        g, H = _ortho(q[b, 1:])
        grad[b, 1:] += s * g
        blocks[b, 1:, 1:] += s * H
    return blocks, grad


def body_energy(q, qt, M, volume, stiffness, fixed, h2):
    """affine_body_dynamics.py:193-217: (inertia, orthogonality) in double."""
    q = np.asarray(q, np.float64).reshape(-1, 4, 3)
    qt = np.asarray(qt, np.float64).reshape(-1, 4, 3)
    inertia = ortho = 0.0
    for b in range(len(q)):
        if fixed[b]:
            continue
        d = q[b] - qt[b]
        inertia += 0.5 * float(np.einsum("ik,ij,jk->", d, M[b], d))
        a = q[b, 1:]
        oe = sum((a[i] @ a[i] - 1.0) ** 2 for i in range(3))
        oe += sum(2.0 * (a[i] @ a[j]) ** 2 for i in range(3) for j in range(i + 1, 3))
        ortho += stiffness[b] * volume[b] * h2 * oe
    return inertia, ortho


def jacobian(rest, body, nb, fixed=None):
    """Dense d x / d q (3V x 12 nb); columns of fixed bodies zero."""
    V = len(rest)
    J = np.zeros((3 * V, 12 * nb))
    for v in range(V):
        b = body[v]
        if fixed is not None and fixed[b]:
            continue
        w = np.concatenate(([1.0], rest[v]))
        for k in range(4):
            J[3 * v:3 * v + 3, 12 * b + 3 * k:12 * b + 3 * k + 3] = w[k] * np.eye(3)
    return J


def reduce_force(f, rest, body, fixed, nb):
    """affine_body_dynamics.py:144-157."""
    out = np.zeros((nb, 4, 3))
    for v in range(len(rest)):
        b = body[v]
        if fixed[b]:
            continue
        w = np.concatenate(([1.0], rest[v]))
        out[b] += w[:, None] * f[v]
    return out


def reduce_hessian(rows, cols, vals, rest, body, fixed, scale):
    """affine_body_dynamics.py:166-190: 16 triplets per source block."""
    n = len(rows)
    R = np.zeros((n, 16), np.int64)
    C = np.zeros((n, 16), np.int64)
    Vb = np.zeros((n, 16, 3, 3))
    for s in range(n):
        vi, vj = rows[s], cols[s]
        bi, bj = body[vi], body[vj]
        wi = np.concatenate(([1.0], rest[vi]))
        wj = np.concatenate(([1.0], rest[vj]))
        for a in range(4):
            for c in range(4):
                R[s, 4 * a + c] = 4 * bi + a
                C[s, 4 * a + c] = 4 * bj + c
                if not (fixed[bi] or fixed[bj]):
                    Vb[s, 4 * a + c] = scale * wi[a] * wj[c] * vals[s]
    return R.ravel(), C.ravel(), Vb.reshape(-1, 3, 3)


def dense(rows, cols, vals, n_block_rows):
    A = np.zeros((3 * n_block_rows, 3 * n_block_rows))
    for r, c, v in zip(rows, cols, vals):
        A[3 * r:3 * r + 3, 3 * c:3 * c + 3] += v
    return A


def system(p: on.Problem, q, qt, M, volume, stiffness, fixed, rest, x=None):
    """Gradient (4 nb, 3) and dense matrix (12 nb)^2 of one ABD Newton
    iteration (affine_body_dynamics.py:427-505): body terms plus the IPC
    contact force and Hessian at x = map(q), reduced to affine DOFs with
    scale h^2.  ``p`` carries the contact data (edges, triangles, body, dhat,
    kappa, h, precision) as for the FEM oracle; ``x`` overrides map(q)."""
    nb = len(volume)
    h2 = p.h * p.h
    blocks, grad = body_system(q, qt, M, volume, stiffness, fixed, h2)
    A = np.zeros((12 * nb, 12 * nb))
    for b in range(nb):
        A[12 * b:12 * b + 12, 12 * b:12 * b + 12] = blocks[b].transpose(0, 2, 1, 3).reshape(12, 12)
    x = (affine_map(q, rest, p.body) if x is None else x).astype(p.dtype)
    ee, pt, l0 = on._contacts(p, x)
    V = len(rest)
    f = np.zeros((V, 3))
    Hv = np.zeros((3 * V, 3 * V))
    for idx, F, H, _ in on._narrow(p, x, ee, pt, l0):
        for k in range(4):
            np.add.at(f, idx[:, k], F[:, 3 * k:3 * k + 3])
        for r in range(len(idx)):
            dofs = (3 * idx[r][:, None] + np.arange(3)).reshape(-1)
            Hv[np.ix_(dofs, dofs)] += H[r]
    J = jacobian(rest, p.body, nb, fixed)
    A += h2 * (J.T @ Hv @ J)
    grad = grad.reshape(-1, 3) - h2 * reduce_force(f, rest, p.body, fixed, nb).reshape(-1, 3)
    return grad, A, len(ee), len(pt)


def energy(p: on.Problem, q, qt, M, volume, stiffness, fixed, rest, x=None):
    """Incremental potential of affine_body_dynamics.py:648-663: inertia +
    orthogonality + h^2 * barrier at x = map(q)."""
    inertia, ortho = body_energy(q, qt, M, volume, stiffness, fixed, p.h * p.h)
    x = (affine_map(q, rest, p.body) if x is None else x).astype(p.dtype)
    ee, pt, l0 = on._contacts(p, x)
    barrier = sum(float(E.sum()) for _, _, _, E in on._narrow(p, x, ee, pt, l0))
    return inertia + ortho + p.h * p.h * barrier
