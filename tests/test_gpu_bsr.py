"""BSR assembly against scipy (gpu)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200.bsr import bsr_from_triplets, bsr_mv, scipy_from_triplets

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_trip,nrow", [(0, 5), (1, 1), (1000, 50), (200_000, 30_000), (70_000, 100_000)])
@pytest.mark.parametrize("fp64", [False, True])
def test_bsr_from_triplets(cuda, n_trip, nrow, fp64):
    rng = np.random.default_rng(n_trip + nrow)
    dt = np.float64 if fp64 else np.float32
    rows = rng.integers(0, nrow, size=n_trip).astype(np.int32)
    cols = np.clip(rows + rng.integers(-3, 4, size=n_trip), 0, nrow - 1).astype(np.int32)
    vals = rng.normal(size=(n_trip, 3, 3)).astype(dt)
    if n_trip > 10:
        vals[::9] = 0.0  # pruned
    tr = lambda a: torch.tensor(a, device=cuda)
    A = bsr_from_triplets(nrow, nrow, tr(rows), tr(cols), tr(vals))
    ref = scipy_from_triplets(nrow, nrow, rows, cols, vals)
    got = A.to_scipy().tocsr()
    # pattern: one block per distinct nonzero (row, col)
    keep = np.any(vals != 0, axis=(1, 2))
    uniq = np.unique(rows[keep].astype(np.int64) * nrow + cols[keep])
    assert A.nnz_sync() == len(uniq)
    offs = A.offsets.cpu().numpy()
    assert offs[0] == 0 and offs[-1] == len(uniq) and np.all(np.diff(offs) >= 0)
    colsA = A.columns[: len(uniq)].cpu().numpy()
    for r in range(min(nrow, 200)):
        seg = colsA[offs[r]:offs[r + 1]]
        assert np.all(np.diff(seg) > 0)
    d = (got - ref)
    tol = 1e-12 if fp64 else 1e-5
    assert (abs(d).max() if d.nnz else 0.0) <= tol * max(abs(ref).max() if ref.nnz else 1.0, 1.0)
    # deterministic: same input, same bits
    B = bsr_from_triplets(nrow, nrow, tr(rows), tr(cols), tr(vals))
    assert torch.equal(A.values[: A.nnz_sync()], B.values[: B.nnz_sync()])
    # SpMV
    x = rng.normal(size=(nrow, 3)).astype(dt)
    y = bsr_mv(A, tr(x)).cpu().numpy().ravel()
    yref = ref @ x.ravel().astype(np.float64)
    assert np.abs(y - yref).max() <= (1e-10 if fp64 else 1e-4) * max(np.abs(yref).max(), 1.0)


@pytest.mark.parametrize("lengths", [(1025, 2048, 3000), (5000, 70_000, 4097), (300_000,)])
@pytest.mark.parametrize("fp64", [False, True])
def test_bsr_long_rows(cuda, lengths, fp64):
    """Rows longer than a warp's shared-memory sort (the unknown rows of an
    affine body collect all its contacts) go through the CTA-per-row sort
    and emit; mixed with ordinary short rows."""
    rng = np.random.default_rng(sum(lengths))
    dt = np.float64 if fp64 else np.float32
    nrow = 4000
    rows, cols = [], []
    for k, L in enumerate(lengths):
        r = 7 + 113 * k
        rows.append(np.full(L, r))
        # many duplicate columns, a few runs longer than a warp's slice
        cols.append(np.concatenate([rng.integers(0, nrow, size=L - L // 4), np.full(L // 4, r)]))
    rows.append(rng.integers(0, nrow, size=20_000))
    cols.append(np.clip(rows[-1] + rng.integers(-3, 4, size=20_000), 0, nrow - 1))
    rows = np.concatenate(rows).astype(np.int32)
    cols = np.concatenate(cols).astype(np.int32)
    perm = rng.permutation(len(rows))
    rows, cols = rows[perm], cols[perm]
    vals = rng.normal(size=(len(rows), 3, 3)).astype(dt)
    vals[::11] = 0.0
    tr = lambda a: torch.tensor(a, device=cuda)  # noqa: E731
    A = bsr_from_triplets(nrow, nrow, tr(rows), tr(cols), tr(vals))
    ref = scipy_from_triplets(nrow, nrow, rows, cols, vals)
    keep = np.any(vals != 0, axis=(1, 2))
    uniq = np.unique(rows[keep].astype(np.int64) * nrow + cols[keep])
    assert A.nnz_sync() == len(uniq)
    offs = A.offsets.cpu().numpy()
    colsA = A.columns[: len(uniq)].cpu().numpy()
    for k in range(len(lengths)):
        r = 7 + 113 * k
        assert np.all(np.diff(colsA[offs[r]:offs[r + 1]]) > 0)
    d = A.to_scipy().tocsr() - ref
    tol = 1e-12 if fp64 else 1e-5
    assert (abs(d).max() if d.nnz else 0.0) <= tol * max(abs(ref).max(), 1.0) * (np.sqrt(max(lengths)) / 10 + 1)
    B = bsr_from_triplets(nrow, nrow, tr(rows), tr(cols), tr(vals))
    assert torch.equal(A.values[: A.nnz_sync()], B.values[: B.nnz_sync()])


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("fp64", [False, True])
def test_contact_bsr_equals_generic_assembly(cuda, idx, fp64):
    """The record-structured assembly and the generic triplet assembly give
    the same matrix bit for bit (both sum each block's contributions in
    record order)."""
    from helpers import small_scenes
    from ipc_warp_b200.bsr import contact_bsr
    from test_gpu_dcd import make_solver
    from test_gpu_narrow import run_gpu

    sc = small_scenes()[idx]
    s = make_solver(sc, torch.float64 if fp64 else torch.float32)
    s.detect_collision()
    from ipc_warp_b200.bsr import Triplets
    from ipc_warp_b200.dynamic_contacts import contact_hessian_ee, contact_hessian_pt

    n_ee, n_pt = s.n_contacts, s.n_contacts_pt
    t = Triplets.zeros((n_ee + n_pt) * 16, s.soup.xcs.dtype, s.device)
    b = torch.zeros_like(s.soup.x_transformed)
    contact_hessian_ee(None, s.soup, s.contacts_new, t, b, 1e4, n=n_ee)
    contact_hessian_pt(None, s.soup, s.contacts_pt, t, b, n_ee, 1e4, n=n_pt)
    nv = s.soup.n_verts
    A = bsr_from_triplets(nv, nv, t.rows, t.cols, t.vals)
    B, status = contact_bsr(s.contacts_new, n_ee, s.contacts_pt, n_pt, nv, t)
    assert status == 0
    nnz = A.nnz_sync()
    assert B.nnz_sync() == nnz > 0
    assert torch.equal(A.offsets, B.offsets)
    assert torch.equal(A.columns[:nnz], B.columns[:nnz])
    # same blocks; the generic path sums each run with a warp tree, this one
    # sequentially, so values agree to rounding
    a, bb = A.values[:nnz].double(), B.values[:nnz].double()
    tol = 1e-12 if fp64 else 2e-6
    assert ((a - bb).abs().amax(dim=(1, 2)) <= tol * a.abs().amax(dim=(1, 2)).clamp_min(1e-300)).all()
    # the per-row bucketing takes slots with atomics; the result is the same bits on every run
    C, _ = contact_bsr(s.contacts_new, n_ee, s.contacts_pt, n_pt, nv, t)
    assert torch.equal(B.values[:nnz], C.values[:nnz])


@pytest.mark.parametrize("n_hub,nv", [(256, 40), (257, 40), (3000, 40), (400, 300)])
def test_contact_bsr_long_row(cuda, n_hub, nv):
    """Vertex 0 in n_hub records (one quad each): a long row (its quads sorted
    in shared memory up to 256, past that in the row's own scratch) equals the
    generic assembly; a row with more than 128 distinct columns sets
    IPCB_STATUS_ROW_OVERFLOW (4) so the caller switches to the generic path."""
    from ipc_warp_b200.bsr import Triplets, contact_bsr
    from ipc_warp_b200.contact import Contacts

    rng = np.random.default_rng(n_hub)
    P = n_hub
    recs = np.stack([rng.permutation(np.r_[0, rng.choice(np.arange(1, nv), 3, replace=False)]) for _ in range(P)])
    recs = recs.astype(np.int32)
    vals = rng.normal(size=(P, 4, 4, 3, 3)).astype(np.float32)
    vals[rng.random((P, 4, 4)) < 0.2] = 0.0  # zero blocks are dropped
    mask = (np.abs(vals).reshape(P, 16, 9).max(-1) > 0).astype(np.uint32) @ (1 << np.arange(16, dtype=np.uint32))
    rows = np.repeat(recs, 4, axis=1).reshape(-1)  # triplet 16p + 4ii + jj: row recs[p, ii]
    cols = np.tile(recs, (1, 4)).reshape(-1)       # column recs[p, jj]
    ee = Contacts(P, torch.float32, cuda)
    ee.a1a2b1b2.copy_(torch.tensor(recs))
    ee.cnt.fill_(P)
    pt = Contacts(1, torch.float32, cuda)
    tr = lambda a: torch.tensor(a, device=cuda)
    t = Triplets(tr(rows.astype(np.int32)), tr(cols.astype(np.int32)), tr(vals.reshape(-1, 3, 3)),
                 tr(mask.astype(np.uint16).view(np.int16)))
    B, status = contact_bsr(ee, P, pt, 0, nv, t)
    if nv > 129:
        assert status & 4
        return
    assert status == 0
    A = bsr_from_triplets(nv, nv, t.rows, t.cols, t.vals)
    nnz = A.nnz_sync()
    assert B.nnz_sync() == nnz > 0
    assert torch.equal(A.offsets, B.offsets) and torch.equal(A.columns[:nnz], B.columns[:nnz])
    a, bb = A.values[:nnz].double(), B.values[:nnz].double()
    assert ((a - bb).abs().amax(dim=(1, 2)) <= 2e-5 * a.abs().amax(dim=(1, 2)).clamp_min(1e-30)).all()
    C, _ = contact_bsr(ee, P, pt, 0, nv, t)
    assert torch.equal(B.values[:nnz], C.values[:nnz])
