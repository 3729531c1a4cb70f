"""CPU checks of the oracle itself: its two Hessian routes agree, gradients
match finite differences, barrier derivatives are consistent, predicates
classify hand-built configurations, and the sorted-axis broad phase equals
an O(n^2) enumeration."""
import itertools

import numpy as np
import pytest

from oracle import pyoracle as po


def d2_explicit(kind, P):
    P = np.asarray(P, dtype=np.float64).reshape(4, 3)
    if kind == 0:
        return np.sum((P[0] - P[1]) ** 2)
    if kind == 1:
        e = P[2] - P[1]
        return np.sum(np.cross(P[0] - P[1], e) ** 2) / e.dot(e)
    if kind == 2:
        n = np.cross(P[2] - P[1], P[3] - P[1])
        return (P[0] - P[1]).dot(n) ** 2 / n.dot(n)
    n = np.cross(P[1] - P[0], P[3] - P[2])
    return (P[0] - P[2]).dot(n) ** 2 / n.dot(n)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_gradient_matches_finite_differences(kind):
    rng = np.random.default_rng(kind)
    for _ in range(20):
        P = rng.normal(size=12)
        g, _ = po.feature_dh(kind, P, mode=0)
        h = 1e-6
        fd = np.array([(d2_explicit(kind, P + h * np.eye(12)[i]) - d2_explicit(kind, P - h * np.eye(12)[i])) / (2 * h)
                       for i in range(12)])
        assert np.allclose(g, fd, rtol=1e-6, atol=1e-8)


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_nsd_routes_agree_and_are_nsd(kind):
    rng = np.random.default_rng(10 + kind)
    worst = 0.0
    for _ in range(300):
        P = rng.normal(size=(4, 3))
        if rng.random() < 0.5:  # small distances, as in contact
            if kind == 2:
                P[0] = P[1] + 0.3 * (P[2] - P[1]) + 0.2 * (P[3] - P[1])
                P[0] += 1e-3 * np.cross(P[2] - P[1], P[3] - P[1])
            if kind == 3:
                P[2] = P[0] + 0.4 * (P[1] - P[0]) + 1e-3 * rng.normal(size=3)
        g0, h0 = po.feature_dh(kind, P, mode=0)
        g1, h1 = po.feature_dh(kind, P, mode=1)
        assert np.allclose(g0, g1, rtol=1e-10, atol=1e-12 * np.abs(g0).max())
        scale = max(np.abs(h0).max(), 1e-300)
        worst = max(worst, np.abs(h0 - h1).max() / scale)
        assert np.linalg.eigvalsh(h0).max() <= 1e-10 * scale
    assert worst < 1e-8


def test_nsd_is_negative_part_of_full_hessian():
    """mode 0: H_full - NSD is PSD and NSD is NSD, for a point near a plane."""
    rng = np.random.default_rng(3)
    P = rng.normal(size=(4, 3))
    P[0] = P[1] + 0.25 * (P[2] - P[1]) + 0.25 * (P[3] - P[1]) + 0.01 * np.cross(P[2] - P[1], P[3] - P[1])
    _, nsd = po.feature_dh(2, P, mode=0)
    h = 1e-4
    H = np.zeros((12, 12))
    f = lambda q: d2_explicit(2, q)
    p = P.ravel()
    E = np.eye(12)
    for i in range(12):
        for j in range(12):
            H[i, j] = (f(p + h * E[i] + h * E[j]) - f(p + h * E[i] - h * E[j]) - f(p - h * E[i] + h * E[j])
                       + f(p - h * E[i] - h * E[j])) / (4 * h * h)
    w = np.linalg.eigvalsh(H)
    assert np.linalg.eigvalsh(nsd).min() == pytest.approx(w.min(), rel=1e-3)
    assert np.linalg.eigvalsh(H - nsd).min() > -1e-5 * np.abs(H).max()


def test_barrier_derivatives():
    xh = 1e-6
    x = np.linspace(0.05, 0.95, 37) * xh
    b = po.barrier(x, xh, 1e4)
    h = 1e-6 * xh
    bp = po.barrier(x + h, xh, 1e4)
    bm = po.barrier(x - h, xh, 1e4)
    assert np.allclose(b[:, 1], (bp[:, 0] - bm[:, 0]) / (2 * h), rtol=1e-5)
    assert np.allclose(b[:, 2], (bp[:, 1] - bm[:, 1]) / (2 * h), rtol=1e-5)
    assert np.all(b[:, 0] > 0) and np.all(b[:, 1] < 0) and np.all(b[:, 2] > 0)
    assert np.all(po.barrier(np.array([xh, 2 * xh]), xh, 1e4) == 0)


def test_closest_point_triangle_regions():
    a, b, c = np.array([0, 0, 0.0]), np.array([1, 0, 0.0]), np.array([0, 1, 0.0])
    cases = {
        0: [-0.5, -0.5, 0.1], 1: [1.5, -0.2, 0.1], 2: [-0.2, 1.5, 0.1], 3: [0.5, -0.5, 0.1],
        4: [-0.5, 0.5, 0.1], 5: [0.8, 0.8, 0.1], 6: [0.2, 0.2, 0.1],
    }
    for ty, p in cases.items():
        uvd, t = po.closest_point_triangle(np.array(p), a, b, c)
        assert t[0] == ty
    uvd, t = po.closest_point_triangle(np.array([0.2, 0.3, 0.5]), a, b, c)
    assert uvd[0, 2] == pytest.approx(0.5) and uvd[0, 0] == pytest.approx(0.5) and uvd[0, 1] == pytest.approx(0.2)


def test_closest_point_edge_edge():
    r = po.closest_point_edge_edge(np.array([0, 0, 0.0]), np.array([1, 0, 0.0]), np.array([0.5, -1, 1.0]),
                                   np.array([0.5, 1, 1.0]))
    assert np.allclose(r[0], [0.5, 0.5, 1.0])
    r = po.closest_point_edge_edge(np.array([0, 0, 0.0]), np.array([1, 0, 0.0]), np.array([2, 0, 1.0]),
                                   np.array([3, 0, 1.0]))
    assert np.allclose(r[0], [1.0, 0.0, np.sqrt(2)])


def _brute(x, prims, body, th, kind, exclude=False):
    x32 = x.astype(np.float32)
    out = []
    l0 = np.float32(th) * np.float32(2.0)
    if kind == "ee":
        E = prims.reshape(-1, 2)
        for i, j in itertools.combinations(range(len(E)), 2):
            a1, a2 = E[i]
            b1, b2 = E[j]
            if len({a1, a2} & {b1, b2}) or (exclude and body[a1] == body[b1]):
                continue
            d = po.closest_point_edge_edge(x32[a1], x32[a2], x32[b1], x32[b2])[0, 2]
            if d < l0:
                out.append([a1, a2, b1, b2, i, j])
    else:
        T = prims.reshape(-1, 3)
        for i in range(len(x)):
            for j, t in enumerate(T):
                if i in t or (exclude and body[i] == body[t[0]]):
                    continue
                d = po.closest_point_triangle(x32[i], x32[t[0]], x32[t[1]], x32[t[2]])[0][0, 2]
                if d < l0:
                    out.append([i, t[1], t[0], t[2], i, j])
    return out


def test_broad_phase_equals_quadratic_enumeration():
    from helpers import sort_records
    from ipc_warp_b200 import scenes

    sc = scenes.two_cubes(n=3, gap=3e-4, seed=2)
    for exclude in (False, True):
        ee = sort_records(po.dcd_ee(sc.x, sc.edges, sc.body, sc.thickness, exclude))
        pt = sort_records(po.dcd_pt(sc.x, sc.triangles, sc.body, sc.thickness, exclude))
        assert len(ee) and len(pt)
        assert np.array_equal(ee, sort_records(_brute(sc.x, sc.edges, sc.body, sc.thickness, "ee", exclude)))
        assert np.array_equal(pt, sort_records(_brute(sc.x, sc.triangles, sc.body, sc.thickness, "pt", exclude)))


def test_cubic_constructed_roots():
    rng = np.random.default_rng(0)
    r = np.sort(rng.uniform(0.01, 0.99, size=(200, 3)), axis=1)
    coef = np.stack([-r.prod(1), r[:, 0] * r[:, 1] + r[:, 0] * r[:, 2] + r[:, 1] * r[:, 2], -r.sum(1),
                     np.ones(200)], 1) * 3.0
    nr, roots, st = po.cubic_roots(coef, 0.0, 1.0)
    assert st == 0
    sep = np.diff(r, axis=1).min(1) > 1e-3
    assert np.all(nr[sep] == 3)
    assert np.allclose(roots[sep], r[sep], atol=1e-8)


def test_known_tois():
    p0 = np.array([[0.2, 0.2, 1.0], [0, 0, 0], [1, 0, 0], [0, 1, 0]])
    p1 = p0.copy()
    p1[0, 2] = -1.0
    assert po.collision_time("pt", p0[None], p1[None])[0] == pytest.approx(0.5, abs=1e-9)
    p1[0, :2] = [2.0, 2.0]  # passes beside the triangle
    p1[0, 2] = 1.0
    assert po.collision_time("pt", p0[None], p1[None])[0] == 1.0
    e0 = np.array([[0.0, 0.5, 1.0], [1.0, 0.5, 1.0], [0.5, 0.0, 0.0], [0.5, 1.0, 0.0]])
    e1 = e0.copy()
    e1[:2, 2] = -3.0
    assert po.collision_time("ee", e0[None], e1[None])[0] == pytest.approx(0.25, abs=1e-9)


def test_contact_bsr_equals_scipy_assembly():
    """The oracle's contact BSR (the CPU baseline's assembly stage) equals
    scipy's assembly of the records' 16 triplets, all-zero blocks dropped."""
    import scipy.sparse as sp

    from ipc_warp_b200.bsr import scipy_from_triplets

    rng = np.random.default_rng(0)
    nv, n = 60, 400
    idx = rng.integers(0, nv, (n, 4)).astype(np.int32)
    H = rng.normal(size=(n, 12, 12))
    H[::7] = 0.0
    H[3, 0:3, 3:6] = 0.0
    off, cols, vals = po.contact_bsr(nv, idx, H)
    rows = np.repeat(idx, 4, axis=1).ravel()
    cc = np.tile(idx, (1, 4)).ravel()
    blocks = H.reshape(n, 4, 3, 4, 3).transpose(0, 1, 3, 2, 4).reshape(-1, 3, 3)
    keep = np.any(blocks != 0, axis=(1, 2))
    assert len(cols) == len(np.unique(rows[keep].astype(np.int64) * nv + cc[keep]))
    got = sp.bsr_matrix((vals, cols, off), shape=(3 * nv, 3 * nv))
    ref = scipy_from_triplets(nv, nv, rows, cc, blocks)
    assert abs(got - ref).max() <= 1e-13 * abs(ref).max()
    for r in range(nv):
        assert np.all(np.diff(cols[off[r]:off[r + 1]]) > 0)


def _crossings_brute(x, edges, tris):
    """All E x T pairs, numpy, the same orientation expressions."""
    E = edges.reshape(-1, 2)
    T = tris.reshape(-1, 3)

    def orient(a, b, c, d):
        u, v, w = b - a, c - a, d - a
        cx = v[..., 1] * w[..., 2] - v[..., 2] * w[..., 1]
        cy = v[..., 2] * w[..., 0] - v[..., 0] * w[..., 2]
        cz = v[..., 0] * w[..., 1] - v[..., 1] * w[..., 0]
        return (u[..., 0] * cx + u[..., 1] * cy) + u[..., 2] * cz

    P, Q = x[E[:, 0]][:, None], x[E[:, 1]][:, None]
    A, B, C = x[T[:, 0]][None], x[T[:, 1]][None], x[T[:, 2]][None]
    o1, o2 = orient(A, B, C, P), orient(A, B, C, Q)
    s1, s2, s3 = orient(P, Q, A, B), orient(P, Q, B, C), orient(P, Q, C, A)
    hit = (((o1 > 0) & (o2 < 0)) | ((o1 < 0) & (o2 > 0))) & (((s1 > 0) & (s2 > 0) & (s3 > 0)) |
                                                         ((s1 < 0) & (s2 < 0) & (s3 < 0)))
    shared = (E[:, None, :, None] == T[None, :, None, :]).any(axis=(2, 3))
    hit &= ~shared
    return np.argwhere(hit).astype(np.int32)


def test_edge_triangle_crossings_match_brute_force():
    from ipc_warp_b200 import scenes

    sc = scenes.two_cubes(n=3, gap=1e-3, angle_deg=20.0, seed=1)
    n, pairs = po.edge_triangle_crossings(sc.x, sc.edges, sc.triangles)
    assert n == 0 and len(_crossings_brute(sc.x, sc.edges, sc.triangles)) == 0
    x = sc.x.copy()
    x[sc.body == 1, 1] -= 0.15  # the upper cube sinks into the lower one
    ref = _crossings_brute(x, sc.edges, sc.triangles)
    n, pairs = po.edge_triangle_crossings(x, sc.edges, sc.triangles)
    assert n == len(ref) > 20
    assert np.array_equal(pairs, ref[np.lexsort(ref.T[::-1])])
