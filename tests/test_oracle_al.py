"""The augmented-Lagrangian oracle (oracle/al.py) on hand-made cases: a
vertex falling through a triangle gives one PT record with the analytic
time, the hash matches the reference formula, and merge keeps exactly the
live old keys plus the new ones."""
import numpy as np

from oracle import al


def test_point_through_triangle_record():
    x0 = np.array([[0.2, 0.2, 1.0], [0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    x1 = x0.copy()
    x1[0, 2] = -1.0
    edges = np.array([[1, 2], [2, 3], [3, 1]])
    tris = np.array([[1, 2, 3]])
    body = np.array([0, 1, 1, 1])
    ee, ee_t, pt, pt_t, toi = al.new_intersections(x0, x1, edges, tris, body)
    assert len(ee) == 0 and len(pt) == 1
    assert list(pt[0]) == [0, 1, 2, 3, 0, 0]
    assert abs(pt_t[0] - 0.5) < 1e-9 and abs(toi - 0.5) < 1e-9


def test_hash_pos_wraps_like_int32():
    # (e0 * 73856093) overflows 32 bits for e0 >= 30: wrap, then |v| mod T
    for e0, e1 in [(0, 0), (3, 5), (30, 7), (123456, 654321), (2 ** 20, 2 ** 21)]:
        w = ((e0 * 73856093) & 0xFFFFFFFF) ^ ((e1 * 19349663) & 0xFFFFFFFF)
        w = w - 2 ** 32 if w >= 2 ** 31 else w
        assert al.hash_pos(e0, e1, 97) == abs(w) % 97


def test_create_and_merge():
    recs = np.array([[0, 1, 2, 3, 0, 5], [2, 3, 4, 5, 1, 6], [6, 7, 8, 9, 2, 7]])
    alpha = np.array([0.5, 0.2, 0.9])
    vt = al.vertex_toi(recs, alpha, 10)
    assert vt[0] == 0.5 and vt[2] == 0.2 and vt[9] == 0.9
    h = al.create(recs, alpha, vt, 8)
    keys = sorted(k for v in h.values() for k in v)
    # record 0: its vertices 0 and 1 have toi 0.5 -> kept; all are kept here
    assert keys == [(0, 5), (1, 6), (2, 7)]
    m = al.merge([(0, 5), (1, 6)], [0.5, 0.001], [(1, 6), (2, 7)], 8)
    assert sorted(k for v in m.values() for k in v) == [(0, 5), (2, 7)]
