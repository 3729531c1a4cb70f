"""Narrow phase: per-record force, 12x12 Hessian and energy against the CPU
oracle (independent hyper-dual + Jacobi route).  Tolerances: 1e-5 relative
(per record, normwise) in float32 mode, 1e-10 in float64 mode (gpu)."""
import numpy as np
import pytest
import torch

from helpers import rel_err, small_scenes
from oracle import pyoracle as po
from test_gpu_dcd import make_solver

pytestmark = pytest.mark.gpu

TOL = {False: 1e-5, True: 1e-10}


def run_gpu(s, kappa):
    from ipc_warp_b200.bsr import Triplets
    from ipc_warp_b200.dynamic_contacts import (contact_energy_ee, contact_energy_pt, contact_hessian_ee,
                                                contact_hessian_pt)

    dtype = s.soup.xcs.dtype
    n_ee, n_pt = s.n_contacts, s.n_contacts_pt
    t = Triplets.zeros((n_ee + n_pt) * 16, dtype, s.device)
    b = torch.zeros_like(s.soup.x_transformed)
    contact_hessian_ee(None, s.soup, s.contacts_new, t, b, kappa, n=n_ee)
    contact_hessian_pt(None, s.soup, s.contacts_pt, t, b, n_ee, kappa, n=n_pt)
    e_ee = torch.zeros(1, dtype=torch.float64, device=s.device)
    e_pt = torch.zeros(1, dtype=torch.float64, device=s.device)
    contact_energy_ee(None, s.soup, s.contacts_new, e_ee, kappa, n=n_ee)
    contact_energy_pt(None, s.soup, s.contacts_pt, e_pt, kappa, n=n_pt)
    return (t.rows.cpu().numpy(), t.cols.cpu().numpy(), t.vals.cpu().numpy().astype(np.float64),
            b.cpu().numpy().astype(np.float64), float(e_ee.item()), float(e_pt.item()))


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("fp64", [False, True])
def test_narrow_matches_oracle(cuda, idx, fp64):
    sc = small_scenes()[idx]
    kappa = 1e4
    s = make_solver(sc, torch.float64 if fp64 else torch.float32)
    s.detect_collision()
    rows, cols, vals, b, e_ee, e_pt = run_gpu(s, kappa)
    xs = s.soup.x_transformed.cpu().numpy()
    xr = s.soup.xcs.cpu().numpy()
    tol = TOL[fp64]
    b_ref = np.zeros_like(xs, dtype=np.float64)
    offset = 0
    for kind, L, n, e_gpu in (("ee", s.contacts_new, s.n_contacts, e_ee), ("pt", s.contacts_pt, s.n_contacts_pt, e_pt)):
        idx4 = L.a1a2b1b2[:n].cpu().numpy()
        l0 = L.l0[:n].cpu().numpy()
        F, H, E, act = po.narrow(kind, idx4, l0, xs, xr, kappa, fp64=fp64, mode=0)
        assert act.sum() > 0
        worst = 0.0
        for p in range(n):
            base = (offset + p) * 16
            blk = vals[base:base + 16]
            Hg = np.zeros((12, 12))
            for ii in range(4):
                for jj in range(4):
                    Hg[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3] = blk[ii * 4 + jj]
                    if act[p]:
                        assert rows[base + ii * 4 + jj] == idx4[p][ii]
                        assert cols[base + ii * 4 + jj] == idx4[p][jj]
            if not act[p]:
                assert not np.any(Hg) and not np.any(rows[base:base + 16])
                continue
            worst = max(worst, rel_err(Hg, H[p]))
            for k in range(4):
                b_ref[idx4[p][k]] += F[p, 3 * k:3 * k + 3]
        assert worst <= tol, (kind, worst)
        assert abs(e_gpu - E.sum()) <= tol * max(abs(E.sum()), 1e-300), (kind, e_gpu, E.sum())
        offset += n
    assert rel_err(b, b_ref) <= tol


def test_hessian_is_psd_and_symmetric(cuda):
    sc = small_scenes()[0]
    s = make_solver(sc, torch.float64)
    s.detect_collision()
    rows, cols, vals, b, _, _ = run_gpu(s, 1e4)
    n = s.n_contacts + s.n_contacts_pt
    for p in range(n):
        H = np.zeros((12, 12))
        for ii in range(4):
            for jj in range(4):
                H[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3] = vals[p * 16 + ii * 4 + jj]
        if not np.any(H):
            continue
        assert np.allclose(H, H.T, rtol=0, atol=1e-12 * np.abs(H).max())
        assert np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("fp64", [False, True])
def test_class_sorted_path_equals_per_cta_path(cuda, idx, fp64):
    """ipcb_contact_hessian_sorted (records in cost-class order over the whole
    list) writes the same blocks, rows, columns and masks as the per-CTA
    ordering, bit for bit; the force differs only by the order of its
    atomics; its order array is a permutation of the records."""
    from ipc_warp_b200 import _native as N
    from ipc_warp_b200.bsr import Triplets
    from ipc_warp_b200.dynamic_contacts import contact_hessian_ee, contact_hessian_pt, hessian_workspace

    sc = small_scenes()[idx]
    dtype = torch.float64 if fp64 else torch.float32
    s = make_solver(sc, dtype)
    s.detect_collision()
    n_ee, n_pt = s.n_contacts, s.n_contacts_pt
    out = []
    for sorted_path in (False, True):
        t = Triplets.zeros((n_ee + n_pt) * 16, dtype, s.device)
        b = torch.zeros_like(s.soup.x_transformed)
        ws_ee = hessian_workspace(s.contacts_new, None) if sorted_path else None
        ws_pt = hessian_workspace(s.contacts_pt, None) if sorted_path else None
        contact_hessian_ee(None, s.soup, s.contacts_new, t, b, 1e4, n=n_ee, ws=ws_ee)
        contact_hessian_pt(None, s.soup, s.contacts_pt, t, b, n_ee, 1e4, n=n_pt, ws=ws_pt)
        torch.cuda.synchronize()
        out.append((t, b))
        if sorted_path:
            for ws, n, L in ((ws_ee, n_ee, s.contacts_new), (ws_pt, n_pt, s.contacts_pt)):
                cap = L.capacity
                off = 256 + ((cap * 16 + 255) // 256) * 256
                order = ws[off:off + 4 * n].view(torch.int32).cpu().numpy()
                assert np.array_equal(np.sort(order), np.arange(n))
                counts = ws[:16].view(torch.int32).cpu().numpy()
                assert counts.sum() == n
    (ta, ba), (tb, bb) = out
    assert torch.equal(ta.rows, tb.rows) and torch.equal(ta.cols, tb.cols)
    assert torch.equal(ta.vals, tb.vals) and torch.equal(ta.mask, tb.mask)
    tol = TOL[fp64]
    assert rel_err(bb.double().cpu().numpy(), ba.double().cpu().numpy()) <= tol
    assert N.size("ipcb_contact_hessian_workspace", 1000) >= 256 + 1000 * 20
