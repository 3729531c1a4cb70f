"""Augmented-Lagrangian CCD lists (new_intersections) and the hashed active
set against oracle/al.py (gpu)."""
import numpy as np
import pytest
import torch

from helpers import small_scenes
from ipc_warp_b200 import contact
from ipc_warp_b200.active_set import ActiveSet, accumulate_vertex_toi
from ipc_warp_b200.contact import ContactSolverBase, Soup
from oracle import al

pytestmark = pytest.mark.gpu


def _solver(sc, dtype):
    class S(ContactSolverBase):
        def __init__(self):
            contact._thickness = sc.thickness
            contact.buffer = sc.thickness
            self.soup = Soup.from_numpy(sc.x, sc.edges, sc.triangles, sc.body, xcs=sc.xcs, dtype=dtype)
            ContactSolverBase.__init__(self)

    return S()


def _motion(sc, seed):
    """x1 = x0 - dx: body 1 moves through body 0's surface (several dhat)."""
    rng = np.random.default_rng(seed)
    dx = np.zeros_like(sc.x)
    dx[sc.body == 1] += np.array([0.0, 3.0, 0.0]) * sc.dhat
    dx += rng.normal(scale=0.3 * sc.dhat, size=dx.shape)
    return sc.x - dx


def _records(lst, n):
    r = torch.cat([lst.a1a2b1b2[:n], lst.e0e1[:n]], dim=1).cpu().numpy().astype(np.int64)
    a = lst.alpha[:n].double().cpu().numpy()
    order = np.lexsort(r.T[::-1])
    return r[order], a[order]


def _sorted(rec, t):
    order = np.lexsort(rec.T[::-1])
    return rec[order], t[order]


@pytest.mark.parametrize("idx", [0, 1])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_new_intersections_match_oracle(cuda, idx, dtype):
    sc = small_scenes()[idx]
    s = _solver(sc, dtype)
    x1 = _motion(sc, idx)
    x0t = torch.tensor(sc.x, dtype=dtype, device=cuda)
    x1t = torch.tensor(x1, dtype=dtype, device=cuda)
    alpha = s.new_intersections(x0t, x1t)
    assert s.status == 0
    x0h, x1h = x0t.double().cpu().numpy(), x1t.double().cpu().numpy()
    ee, ee_t, pt, pt_t, toi = al.new_intersections(x0h, x1h, sc.edges, sc.triangles, sc.body)
    assert len(ee) > 0 and len(pt) > 0
    got_ee, a_ee = _records(s.contacts_new, s.n_contacts)
    got_pt, a_pt = _records(s.contacts_pt, s.n_contacts_pt)
    ee, ee_t = _sorted(ee, ee_t)
    pt, pt_t = _sorted(pt, pt_t)
    assert np.array_equal(got_ee, ee) and np.array_equal(got_pt, pt)
    if dtype == torch.float64:
        assert np.array_equal(a_ee, ee_t) and np.array_equal(a_pt, pt_t)
        assert alpha == pytest.approx(0.9 * toi, rel=1e-15)
    else:  # times rounded toward zero to float
        for a, t in ((a_ee, ee_t), (a_pt, pt_t)):
            assert np.all(a <= t) and np.all(t - a <= 2.0 ** -23 * t + 1e-45)
    l0 = s.contacts_new.l0[: s.n_contacts].double().cpu().numpy()
    th = np.float64(np.float32(sc.thickness)) if dtype == torch.float32 else sc.thickness
    assert np.all(l0 == (np.float32(th) * np.float32(2) if dtype == torch.float32 else th * 2.0))


def test_new_intersections_grow_lists(cuda):
    sc = small_scenes()[0]
    old = contact.contact_volume
    contact.contact_volume = 2
    try:
        s = _solver(sc, torch.float64)
    finally:
        contact.contact_volume = old
    x1 = _motion(sc, 0)
    s.new_intersections(torch.tensor(sc.x, dtype=torch.float64, device=cuda),
                        torch.tensor(x1, dtype=torch.float64, device=cuda))
    ee, _, pt, _, _ = al.new_intersections(sc.x, x1, sc.edges, sc.triangles, sc.body)
    assert s.n_contacts == len(ee) > 2 and s.contacts_new.capacity >= len(ee)
    assert s.n_contacts_pt == len(pt)


def _bucket_keys(h):
    start = h.cell_start.cpu().numpy()
    keys = h.e0e1.cpu().numpy()
    out = {}
    for b in range(h.table_size):
        if start[b + 1] > start[b]:
            out[b] = sorted(map(tuple, keys[start[b]:start[b + 1]].tolist()))
    return out


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_active_set_create_and_merge(cuda, dtype):
    sc = small_scenes()[1]
    s = _solver(sc, dtype)
    x1 = _motion(sc, 7)
    s.new_intersections(torch.tensor(sc.x, dtype=dtype, device=cuda), torch.tensor(x1, dtype=dtype, device=cuda))
    n = s.n_contacts
    rec, alpha = _records(s.contacts_new, n)
    vt = torch.ones(s.soup.n_verts, dtype=dtype, device=cuda)
    accumulate_vertex_toi(s.contacts_new, n, vt)
    vt_ref = al.vertex_toi(rec, alpha, s.soup.n_verts)
    assert np.array_equal(vt.double().cpu().numpy(), vt_ref)
    A = ActiveSet(4, dtype=dtype, device=cuda)
    A.create_hash(s.contacts_new, n, vt)
    ref = al.create(rec, alpha, vt.double().cpu().numpy(), A.hash.table_size)
    assert A.count() == sum(len(v) for v in ref.values()) > 0
    assert _bucket_keys(A.hash) == ref
    k = A.count()
    assert torch.all(A.hash.gamma[:k] == 1) and torch.all(A.hash.lam[:k] == 0) and torch.all(A.hash.mollifier[:k] == 1)
    # age half of the old set below the decay threshold, then merge a second set
    A.hash.gamma[: k // 2] = 0.001
    old_keys = A.hash.e0e1[:k].cpu().numpy().tolist()
    old_gamma = A.hash.gamma[:k].double().cpu().numpy()
    s.new_intersections(torch.tensor(sc.x, dtype=dtype, device=cuda),
                        torch.tensor(_motion(sc, 8), dtype=dtype, device=cuda))
    B = ActiveSet(4, dtype=dtype, device=cuda)
    vt2 = torch.ones_like(vt)
    accumulate_vertex_toi(s.contacts_new, s.n_contacts, vt2)
    B.create_hash(s.contacts_new, s.n_contacts, vt2)
    new_keys = B.hash.e0e1[: B.count()].cpu().numpy().tolist()
    A.merge(B)
    ref = al.merge(old_keys, old_gamma, new_keys, A.hash.table_size)
    assert _bucket_keys(A.hash) == ref


def test_new_intersections_with_a_small_candidate_list(cuda):
    """The in-place pass (taken when staged candidates overflow) appends each
    colliding pair once, as the staged pass does."""
    sc = small_scenes()[0]
    s = _solver(sc, torch.float64)
    x0 = torch.tensor(sc.x, dtype=torch.float64, device=cuda)
    x1 = torch.tensor(_motion(sc, 3), dtype=torch.float64, device=cuda)
    a_full = s.new_intersections(x0, x1)
    ee_full, _ = _records(s.contacts_new, s.n_contacts)
    pt_full, _ = _records(s.contacts_pt, s.n_contacts_pt)
    from ipc_warp_b200 import _native as N

    s._toi_ws = torch.empty(N.size("ipcb_toi_workspace", 8), dtype=torch.uint8, device=cuda)  # 8 staged pairs
    a_small = s.new_intersections(x0, x1)
    assert a_small == a_full
    assert np.array_equal(_records(s.contacts_new, s.n_contacts)[0], ee_full)
    assert np.array_equal(_records(s.contacts_pt, s.n_contacts_pt)[0], pt_full)
