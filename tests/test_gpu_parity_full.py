"""Parity at the benchmark's size (gpu).

One ``ContactPipeline.iteration`` -- the benchmark's step -- on the full
workloads, every output checked against the CPU oracle on the same inputs:

* the screw-and-nut configuration (60-degree thread, pitch 0.1, 12 turns,
  about 0.5M surface triangles per body, the nut loaded onto one flank,
  about 345k candidate pairs) with the driven nut's step: the bench workload;
* the rod-twist bundle in its wound contact state (16 rods of 4x4x256 hex
  cells, 102,800 vertices, about 739k candidate pairs): the second bench line;
* the two-cube configuration exactly as generated (8^3 cells per cube,
  upper cube turned 15 degrees about z, 1e-3 above the lower one, jitter
  1e-5, dhat 1e-3, kappa 1e4), and the same scene later in its fall, with
  the upper cube 6e-4 lower so that its lowest edge is inside the barrier.

Checks, with the tolerances of the narrow-phase and CCD tests:

* EE and PT candidate sets bit-exact as sorted record lists;
* every record's 12x12 Hessian (its 16 triplet blocks) within 1e-5 (float32)
  / 1e-10 (float64) normwise of the oracle's, inactive records all zero;
* the assembled force and the barrier energy within the same tolerance;
* the contact BSR: on 3000 sampled rows, every block equals the sum of the
  row's triplets (pattern exact);
* the scene TOI of a seeded Newton direction not above the oracle's and
  within 1e-6 of it.
"""
import functools

import numpy as np
import pytest
import torch

from helpers import sort_records
from ipc_warp_b200 import scenes
from ipc_warp_b200.pipeline import ContactPipeline
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL = {torch.float32: 1e-5, torch.float64: 1e-10}


@functools.lru_cache(maxsize=None)
def workload(name):
    """(scene, Newton direction) of a named workload; x1 = x - dx."""
    if name == "rod_bundle":
        import bench

        sc = bench.scene("rod_bundle")
        return sc, bench.direction(sc)
    if name == "screw_nut":
        sc = scenes.screw_and_nut()  # the screw-and-nut configuration: 0.5M surface triangles per body
        return sc, scenes.screw_direction(sc)
    sc = scenes.two_cubes()  # cfg1 as specified
    rng = np.random.default_rng(11)
    up = sc.body == 1
    if name == "two_cubes_falling":
        sc.x[up, 1] -= 6e-4  # later in the fall: the lowest edge is 4e-4 above the lower cube
    dx = rng.normal(scale=2e-5, size=sc.x.shape)
    dx[up, 1] += 2.0 * sc.meta["gap"]  # the upper cube falls through twice the gap
    return sc, dx


def run(name, dtype, cuda):
    sc, dx = workload(name)
    pipe = ContactPipeline.from_scene(sc, dtype=dtype, device=cuda)
    dxt = torch.tensor(dx, dtype=dtype, device=cuda)
    pipe.iteration(dxt)  # eager pass (list growth), then the captured graph
    res = pipe.iteration(dxt)
    torch.cuda.synchronize()
    return sc, dx, pipe, res


def records_to_hessians(vals, n, offset):
    """(n, 12, 12) from the 16 blocks (slot ii*4+jj) of records offset..offset+n."""
    v = vals[16 * offset:16 * (offset + n)].reshape(n, 4, 4, 3, 3)
    return v.transpose(0, 1, 3, 2, 4).reshape(n, 12, 12)


@pytest.mark.parametrize("name,dtype", [("screw_nut", torch.float32), ("screw_nut", torch.float64),
                                        ("rod_bundle", torch.float32), ("rod_bundle", torch.float64),
                                        ("two_cubes", torch.float32), ("two_cubes_falling", torch.float32),
                                        ("two_cubes_falling", torch.float64)])
def test_full_size_parity(cuda, name, dtype):
    sc, dx, pipe, res = run(name, dtype, cuda)
    fp64 = dtype == torch.float64
    tol = TOL[dtype]
    assert res.status == 0
    # ---- candidate sets, bit-exact (the float32 predicate in both builds)
    x32 = sc.x.astype(np.float32)
    th = np.float32(sc.thickness)
    ee = sort_records(pipe.contacts_new.records(res.n_ee).cpu().numpy())
    pt = sort_records(pipe.contacts_pt.records(res.n_pt).cpu().numpy())
    assert np.array_equal(ee, sort_records(po.dcd_ee(x32, sc.edges, sc.body, th, cap=1 << 21)))
    assert np.array_equal(pt, sort_records(po.dcd_pt(x32, sc.triangles, sc.body, th, cap=1 << 21)))
    assert res.n_ee > 0 and res.n_pt > 0  # the jitter brings parts of the lowest edge inside dhat
    if name == "rod_bundle":
        assert res.n_ee + res.n_pt > 700_000
    if name == "screw_nut":
        assert res.n_ee + res.n_pt > 300_000

    # ---- narrow phase: every record, in chunks
    x = pipe.soup.x_transformed.cpu().numpy()
    xr = pipe.soup.xcs.cpu().numpy()
    t = pipe.collision_triplets
    vals = t.vals.cpu().numpy()
    rows = t.rows.cpu().numpy()
    b_ref = np.zeros(x.shape, np.float64)
    e_ref = 0.0
    offset = 0
    for kind, L, n in (("ee", pipe.contacts_new, res.n_ee), ("pt", pipe.contacts_pt, res.n_pt)):
        idx = L.a1a2b1b2[:n].cpu().numpy()
        l0 = L.l0[:n].cpu().numpy()
        worst = 0.0
        for a in range(0, n, 100_000):
            m = min(n, a + 100_000) - a
            F, H, E, act = po.narrow(kind, idx[a:a + m], l0[a:a + m], x, xr, sc.kappa, fp64=fp64, mode=0)
            Hg = records_to_hessians(vals, m, offset + a).astype(np.float64)
            on = act.astype(bool)
            assert not np.any(Hg[~on]) and not np.any(rows.reshape(-1, 16)[offset + a:offset + a + m][~on])
            den = np.abs(H[on]).max(axis=(1, 2))
            err = np.abs(Hg[on] - H[on]).max(axis=(1, 2)) / np.where(den > 0, den, 1.0)
            worst = max(worst, float(err.max()) if err.size else 0.0)
            for k in range(4):
                np.add.at(b_ref, idx[a:a + m, k], F[:, 3 * k:3 * k + 3])
            e_ref += float(E.sum())
        assert worst <= tol, (kind, worst)
        offset += n
    b = pipe.b.cpu().numpy().astype(np.float64)
    assert np.abs(b - b_ref).max() <= tol * max(np.abs(b_ref).max(), 1e-300)
    e_gpu = float(pipe._energy.item())
    assert abs(e_gpu - e_ref) <= tol * max(abs(e_ref), 1e-300), (e_gpu, e_ref)

    # ---- contact BSR rows = sums of their triplets
    H = pipe.collision_hessian
    if res.n_ee + res.n_pt:
        offs = H.offsets.cpu().numpy().astype(np.int64)
        cols = H.columns.cpu().numpy()
        hv = H.values.cpu().numpy().astype(np.float64)
        n_rec = res.n_ee + res.n_pt
        tr_rows = rows[:16 * n_rec].astype(np.int64)
        tr_cols = t.cols.cpu().numpy()[:16 * n_rec].astype(np.int64)
        tr_vals = vals[:16 * n_rec].astype(np.float64)
        nz = np.any(tr_vals != 0, axis=(1, 2))
        touched = np.unique(tr_rows[nz])
        # every row without a non-zero contribution is empty (most vertex rows
        # of the screw and nut: the assembly only visits the touched rows)
        untouched = np.ones(offs.size - 1, bool)
        untouched[touched] = False
        assert not np.any(np.diff(offs)[untouched])
        assert offs[-1] == int(H.nnz_sync())
        rng = np.random.default_rng(0)
        sample = set(rng.choice(touched, size=min(3000, touched.size), replace=False).tolist())
        sel = np.nonzero(nz & np.isin(tr_rows, list(sample)))[0]
        sel = sel[np.argsort(tr_rows[sel], kind="stable")]
        starts = np.flatnonzero(np.r_[True, tr_rows[sel][1:] != tr_rows[sel][:-1], True])
        assert starts.size - 1 == len(sample)
        for a, z in zip(starts[:-1], starts[1:]):
            mine = sel[a:z]
            r = tr_rows[mine[0]]
            uc, inv = np.unique(tr_cols[mine], return_inverse=True)
            ref = np.zeros((uc.size, 3, 3))
            np.add.at(ref, inv, tr_vals[mine])
            assert np.array_equal(cols[offs[r]:offs[r + 1]], uc)
            scale = max(np.abs(ref).max(), 1e-300)
            assert np.abs(hv[offs[r]:offs[r + 1]] - ref).max() <= tol * scale

    # ---- TOI of the Newton direction
    x1 = pipe.ccd_x1.cpu().numpy()
    assert np.array_equal(x1, x - dx.astype(x.dtype))
    toi = float(pipe.ccd_toi.item())
    otoi, ost = po.scene_toi(x, x1, sc.edges, sc.triangles, sc.body, fp64=fp64)
    assert ost == 0 and otoi < 1.0
    assert toi <= otoi and otoi - toi <= 1e-6, (toi, otoi)
    assert res.alpha == pytest.approx(0.9 * toi)
