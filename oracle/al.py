"""CPU restatement of the augmented-Lagrangian CCD lists and hashed active
set (test infrastructure only; the product never imports this module).

Follows contact.py:587-670 (new_intersections with edge_edge_intersections /
point_triangle_intersections 371-442 and append_ccd 186-197) and
augmented_lagrangian.py:105-198, 506-572 (accumulate_vertex_toi,
filter_accept, create_hash, merge, hash_pos).  Every pair is tested (brute
force); the per-pair time of impact is the oracle's collision_time.
Parity pin: the per-pair times are the oracle's, which tests/test_golden.py
pins against the reference's own ccd.py on fixtures; the list and hash logic
is restated from the reference lines above.
"""
from __future__ import annotations

import numpy as np

from . import pyoracle as po

TOI_FILTER_EPS = 1e-12
DECAY_THRESHOLD = 0.01


def new_intersections(x0, x1, edges, triangles, body, exclude_same_body=False):
    """(ee records, pt records, toi): records are rows (a1, a2, b1, b2, e0, e1)
    with their times t < 1 (double), toi = min(t, 1)."""
    x0 = np.asarray(x0, np.float64)
    x1 = np.asarray(x1, np.float64)
    E = np.asarray(edges).reshape(-1, 2)
    T = np.asarray(triangles).reshape(-1, 3)
    ne = len(E)
    I, J = np.triu_indices(ne, 1)
    ea, eb = E[I], E[J]
    keep = ~((ea[:, 0] == eb[:, 0]) | (ea[:, 0] == eb[:, 1]) | (ea[:, 1] == eb[:, 0]) | (ea[:, 1] == eb[:, 1]))
    if exclude_same_body:
        keep &= body[ea[:, 0]] != body[eb[:, 0]]
    I, J, ea, eb = I[keep], J[keep], ea[keep], eb[keep]
    ids = np.concatenate([ea, eb], axis=1)
    t = po.collision_time("ee", x0[ids].reshape(-1, 12), x1[ids].reshape(-1, 12)) if len(ids) else np.zeros(0)
    hit = t < 1.0
    ee = np.concatenate([ids[hit], I[hit, None], J[hit, None]], axis=1)
    ee_t = t[hit]
    V = len(x0)
    P, F = np.meshgrid(np.arange(V), np.arange(len(T)), indexing="ij")
    P, F = P.ravel(), F.ravel()
    tri = T[F]
    keep = ~((tri[:, 0] == P) | (tri[:, 1] == P) | (tri[:, 2] == P))
    if exclude_same_body:
        keep &= body[P] != body[tri[:, 0]]
    P, F, tri = P[keep], F[keep], tri[keep]
    ids = np.concatenate([P[:, None], tri], axis=1)
    t2 = po.collision_time("pt", x0[ids].reshape(-1, 12), x1[ids].reshape(-1, 12)) if len(ids) else np.zeros(0)
    hit = t2 < 1.0
    pt = np.concatenate([ids[hit], P[hit, None], F[hit, None]], axis=1)
    pt_t = t2[hit]
    toi = min([1.0] + list(ee_t) + list(pt_t))
    return ee, ee_t, pt, pt_t, toi


def hash_pos(e0, e1, table_size):
    """augmented_lagrangian.py hash_pos in 32-bit wrapping arithmetic."""
    v = (((int(e0) * 73856093) & 0xFFFFFFFF) ^ ((int(e1) * 19349663) & 0xFFFFFFFF))
    if v >= 1 << 31:
        v -= 1 << 32
    if v < 0:
        v = -v
    return v % table_size


def vertex_toi(records, alpha, n_verts, init=1.0):
    out = np.full(n_verts, init)
    for r, a in zip(records, alpha):
        for v in r[:4]:
            out[v] = min(out[v], a)
    return out


def create(records, alpha, vtoi, table_size):
    """Kept entries per bucket: {bucket: sorted list of (e0, e1)}."""
    buckets = {}
    for r, a in zip(records, alpha):
        if any(a <= vtoi[v] + TOI_FILTER_EPS for v in r[:4]):
            key = (int(r[4]), int(r[5]))
            buckets.setdefault(hash_pos(*key, table_size), []).append(key)
    return {b: sorted(k) for b, k in buckets.items()}


def merge(old_keys, old_gamma, new_keys, table_size):
    """Keys of the merged set per bucket: old keys with gamma >= 0.01 and
    new keys not in old."""
    old = set(map(tuple, old_keys))
    out = {}
    for k, g in zip(old_keys, old_gamma):
        if g >= DECAY_THRESHOLD:
            out.setdefault(hash_pos(*k, table_size), []).append(tuple(k))
    for k in new_keys:
        if tuple(k) not in old:
            out.setdefault(hash_pos(*k, table_size), []).append(tuple(k))
    return {b: sorted(v) for b, v in out.items()}
