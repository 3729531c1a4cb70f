"""Broad phase: candidate sets must equal the oracle's bit for bit (gpu)."""
import numpy as np
import pytest
import torch

from helpers import small_scenes, sort_records
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def make_solver(sc, dtype=torch.float32, exclude=False):
    from ipc_warp_b200.contact import ContactSolverBase

    class S(ContactSolverBase):
        def __init__(self):
            from ipc_warp_b200 import contact
            from ipc_warp_b200.contact import Soup

            contact._thickness = sc.thickness
            contact.buffer = sc.thickness
            self.soup = Soup.from_numpy(sc.x, sc.edges, sc.triangles, sc.body, xcs=sc.xcs, dtype=dtype)
            ContactSolverBase.__init__(self)
            self.disable_self_collision = exclude

    return S()


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("exclude", [False, True])
@pytest.mark.parametrize("fp64", [False, True])
def test_candidates_match_oracle(cuda, idx, exclude, fp64):
    sc = small_scenes()[idx]
    s = make_solver(sc, torch.float64 if fp64 else torch.float32, exclude)
    s.detect_collision()
    assert s.status == 0
    ee = sort_records(s.contacts_new.records(s.n_contacts).cpu().numpy())
    pt = sort_records(s.contacts_pt.records(s.n_contacts_pt).cpu().numpy())
    x32 = sc.x.astype(np.float32)
    oee = sort_records(po.dcd_ee(x32, sc.edges, sc.body, np.float32(sc.thickness), exclude))
    opt = sort_records(po.dcd_pt(x32, sc.triangles, sc.body, np.float32(sc.thickness), exclude))
    assert len(oee) > 0 and len(opt) > 0
    assert np.array_equal(ee, oee)
    assert np.array_equal(pt, opt)
    # record scalars: l0 = 2 * thickness, alpha = 1e-6
    l0 = s.contacts_new.l0[: s.n_contacts].cpu().numpy()
    dt = np.float64 if fp64 else np.float32
    assert np.all(l0 == dt(np.float32(sc.thickness)) * dt(2.0))


def test_overflow_grow_and_relaunch(cuda):
    from ipc_warp_b200 import contact

    sc = small_scenes()[0]
    old = contact.contact_volume
    contact.contact_volume = 1
    try:
        s = make_solver(sc)
        s.detect_collision()
    finally:
        contact.contact_volume = old
    assert s.contacts_new.capacity >= s.n_contacts > 1
    assert s.contacts_pt.capacity >= s.n_contacts_pt > 1
    ee = sort_records(s.contacts_new.records(s.n_contacts).cpu().numpy())
    oee = sort_records(po.dcd_ee(sc.x.astype(np.float32), sc.edges, sc.body, np.float32(sc.thickness)))
    assert np.array_equal(ee, oee)


def test_refit_after_motion_keeps_parity(cuda):
    sc = small_scenes()[2]
    s = make_solver(sc)
    s.detect_collision()
    rng = np.random.default_rng(11)
    x2 = sc.x + rng.uniform(-0.2, 0.2, size=sc.x.shape) * sc.dhat
    s.soup.x_transformed.copy_(torch.tensor(x2, dtype=torch.float32))
    s.detect_collision()
    ee = sort_records(s.contacts_new.records(s.n_contacts).cpu().numpy())
    pt = sort_records(s.contacts_pt.records(s.n_contacts_pt).cpu().numpy())
    x32 = x2.astype(np.float32)
    assert np.array_equal(ee, sort_records(po.dcd_ee(x32, sc.edges, sc.body, np.float32(sc.thickness))))
    assert np.array_equal(pt, sort_records(po.dcd_pt(x32, sc.triangles, sc.body, np.float32(sc.thickness))))


def test_no_contacts_and_single_triangle(cuda):
    from ipc_warp_b200 import scenes

    sc = scenes.two_cubes(n=2, gap=0.5)  # far apart
    s = make_solver(sc)
    s.detect_collision()
    assert s.n_contacts == 0 and s.n_contacts_pt == 0
    # one triangle and one far point: a single-leaf BVH
    x = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 1e-4]], dtype=np.float64)
    tri = np.array([0, 1, 2], dtype=np.int32)
    edges = np.array([0, 1, 1, 2, 2, 0], dtype=np.int32)
    body = np.array([0, 0, 0, 1], dtype=np.int32)
    sc1 = scenes.Scene("one_tri", x, x.copy(), edges, tri, body, np.zeros((0, 4), np.int32), dhat=1e-3, kappa=1.0)
    s = make_solver(sc1)
    s.detect_collision()
    assert s.n_contacts_pt == 1
    assert s.contacts_pt.records(1).cpu().numpy().tolist() == [[3, 1, 0, 2, 3, 0]]
