"""FixedBodyContactSolver (fixed_bvh_contacts.py:503-827): the body-local
hierarchies give the same DCD candidate sets as the dynamic query with
same-body pairs excluded, and the same CCD bound, on bodies carried by
random affine frames (gpu)."""
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from helpers import small_scenes, sort_records
from ipc_warp_b200 import contact
from ipc_warp_b200.contact import ContactSolverBase, Soup
from ipc_warp_b200.fixed_bvh_contacts import FixedBodyContactSolver

pytestmark = pytest.mark.gpu


def affine_frames(sc, seed, stretch=0.1, singular_body=None):
    """Per body: x = p + A r with p the centroid and A a random rotation times
    a stretch; returns local rest coordinates r, q (nb, 12) = [p, A columns]
    and the world positions recomputed from them."""
    rng = np.random.default_rng(seed)
    nb = int(sc.body.max()) + 1
    q = np.zeros((nb, 12))
    r = np.zeros_like(sc.x)
    xw = np.zeros_like(sc.x)
    for b in range(nb):
        idx = sc.body == b
        c = sc.x[idx].mean(axis=0)
        R, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        R *= np.sign(np.linalg.det(R))
        A = R @ np.diag(rng.uniform(1 - stretch, 1 + stretch, 3))
        if b == singular_body:
            A = A * 1e-4
        r[idx] = np.linalg.solve(A, (sc.x[idx] - c).T).T
        xw[idx] = c + r[idx] @ A.T
        q[b, :3] = c
        q[b, 3:] = A.T.reshape(-1)
    return r, q, xw


def affine_vertex_step(sc, r, dq):
    """dx_v = dp + dA r_v for x1 = x - dx."""
    dA = dq[:, 3:].reshape(-1, 3, 3).transpose(0, 2, 1)
    return dq[sc.body, :3] + np.einsum("vij,vj->vi", dA[sc.body], r)


def make(sc, r, q, xw, dtype):
    class S(FixedBodyContactSolver):
        def __init__(self):
            contact._thickness = sc.thickness
            contact.buffer = sc.thickness
            self.soup = Soup.from_numpy(xw, sc.edges, sc.triangles, sc.body, xcs=r, dtype=dtype)
            ContactSolverBase.__init__(self)
            self.initialize_fixed_body_bvhs(torch.tensor(q, dtype=dtype, device="cuda"))

    return S()


def canon(rec):
    """EE records as (lower edge first); PT records as they are."""
    rec = np.asarray(rec, dtype=np.int64).reshape(-1, 6).copy()
    sw = rec[:, 4] > rec[:, 5]
    rec[sw] = rec[sw][:, [2, 3, 0, 1, 5, 4]]
    return sort_records(rec)


def dcd_sets(s, fixed):
    if fixed:
        s.detect_collision()
    else:
        s.disable_self_collision = True
        ContactSolverBase.detect_collision(s)
    assert s.status == 0
    ee = canon(s.contacts_new.records(s.n_contacts).cpu().numpy())
    pt = sort_records(s.contacts_pt.records(s.n_contacts_pt).cpu().numpy())
    return ee, pt


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_fixed_dcd_equals_dynamic_without_same_body(cuda, idx, dtype):
    sc = small_scenes()[idx]
    r, q, xw = affine_frames(sc, seed=idx)
    s = make(sc, r, q, xw, dtype)
    fee, fpt = dcd_sets(s, True)
    assert s.fixed_body_pair_count_host >= 1
    dee, dpt = dcd_sets(s, False)
    assert len(dee) > 0 and len(dpt) > 0
    assert np.array_equal(fee, dee)
    assert np.array_equal(fpt, dpt)


@pytest.mark.parametrize("idx", [0, 1, 3])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_fixed_ccd_equals_dynamic(cuda, idx, dtype):
    sc = small_scenes()[idx]
    r, q, xw = affine_frames(sc, seed=10 + idx)
    s = make(sc, r, q, xw, dtype)
    rng = np.random.default_rng(idx)
    nb = q.shape[0]
    # every body moves toward the scene centre by a few dhat and turns a little
    centre = q[:, :3].mean(axis=0)
    dq = np.zeros_like(q)
    d = q[:, :3] - centre
    dq[:, :3] = 4.0 * sc.dhat * d / np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-12)
    dq[:, 3:] = 1e-3 * rng.normal(size=(nb, 9))
    dx = torch.tensor(affine_vertex_step(sc, r, dq), dtype=dtype, device="cuda")
    s.disable_self_collision = True
    s.abd_states = SimpleNamespace(dx=torch.tensor(dq, dtype=dtype, device="cuda"))
    a_fixed = s.collision_free_step(dx)
    assert s.status == 0
    del s.abd_states
    a_dyn = s.collision_free_step(dx)
    assert a_dyn < 1.0
    assert a_fixed == pytest.approx(a_dyn, rel=1e-12, abs=0)


def test_singular_frame_falls_back(cuda):
    sc = small_scenes()[2]
    r, q, xw = affine_frames(sc, seed=4, singular_body=1)
    s = make(sc, r, q, xw, torch.float64)
    fee, fpt = dcd_sets(s, True)
    assert s.disable_self_collision is False
    dee, dpt = dcd_sets(s, False)
    assert np.array_equal(fee, dee) and np.array_equal(fpt, dpt)
