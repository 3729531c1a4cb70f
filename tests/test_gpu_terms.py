"""Batched Newton terms (one persistent work-queue launch over the contact
records, the tets and the affine-body items) and the fixed-pattern assembly against the per-term
kernels and the sort-based assembly; BSR pattern union against numpy;
autotuner bookkeeping (gpu)."""
import numpy as np
import pytest
import torch

from helpers import small_scenes
from ipc_warp_b200 import _native as N
from ipc_warp_b200.newton import FEMContactSolver

pytestmark = pytest.mark.gpu


def _dense(A):
    nnz = int(A.nnz_dev.item())
    off = A.offsets.cpu().numpy()
    cols = A.columns.cpu().numpy()[:nnz]
    vals = A.values[:nnz].double().cpu().numpy()
    n = A.nrow
    D = np.zeros((3 * n, 3 * n))
    rows = np.repeat(np.arange(n), np.diff(off))
    for r, c, v in zip(rows, cols, vals):
        D[3 * r:3 * r + 3, 3 * c:3 * c + 3] += v
    return D, rows, cols


def _solver(sc, dtype, assembly):
    fixed = sc.xcs[:, 1] <= sc.xcs[:, 1].min() + 1e-9
    return FEMContactSolver(sc, material="neo_hookean", E=1e6, nu=0.4, rho=1000.0, h=1e-2, fixed=fixed, dtype=dtype,
                            assembly=assembly)


@pytest.mark.parametrize("idx", [0, 1, 2])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_queue_assembly_equals_generic(cuda, idx, dtype):
    sc = small_scenes()[idx]
    rng = np.random.default_rng(idx)
    x = sc.x + rng.normal(scale=0.05 * sc.dhat, size=sc.x.shape)
    out = {}
    for assembly in ("generic", "queue"):
        s = _solver(sc, dtype, assembly)
        s.states.x.copy_(torch.tensor(x, dtype=dtype))
        A = s.compute_A()
        assert s.n_contacts + s.n_contacts_pt > 0
        out[assembly] = (_dense(A), s.b.double().cpu().numpy().copy(), s.n_contacts, s.n_contacts_pt)
    (Dg, rg, cg), bg, *ng = out["generic"]
    (Dq, rq, cq), bq, *nq = out["queue"]
    assert ng == nq
    # identical pattern, values up to the summation order
    assert np.array_equal(rg, rq) and np.array_equal(cg, cq)
    tol = 1e-5 if dtype == torch.float32 else 1e-12
    assert np.abs(Dq - Dg).max() <= tol * np.abs(Dg).max()
    assert np.abs(bq - bg).max() <= tol * max(np.abs(bg).max(), 1e-30) * 10


def test_bsr_union_matches_numpy(cuda):
    rng = np.random.default_rng(0)
    n = 300

    def pattern(density):
        off = [0]
        cols = []
        for r in range(n):
            c = np.sort(rng.choice(n, size=rng.integers(0, int(density * n) + 1), replace=False))
            cols.extend(c.tolist())
            off.append(len(cols))
        return np.array(off, np.int32), np.array(cols, np.int32)

    ao, ac = pattern(0.05)
    bo, bc = pattern(0.02)
    t = lambda a: torch.tensor(a, dtype=torch.int32, device=cuda)
    cap = len(ac) + len(bc)
    co, crow, ccol, sa, sb = (torch.zeros(k, dtype=torch.int32, device=cuda) for k in (n + 1, cap, cap, cap, cap))
    nnz = torch.zeros(1, dtype=torch.int32, device=cuda)
    st = torch.zeros(1, dtype=torch.int32, device=cuda)
    ws = torch.empty(N.size("ipcb_bsr_union_workspace", n), dtype=torch.uint8, device=cuda)
    dao, dac, dbo, dbc = t(ao), t(ac), t(bo), t(bc)  # keep the inputs alive until the launch
    N.call("ipcb_bsr_union", n, N.ptr(dao), N.ptr(dac), N.ptr(dbo), N.ptr(dbc), N.ptr(co), N.ptr(crow),
           N.ptr(ccol), N.ptr(sa), N.ptr(sb), cap, N.ptr(nnz), N.ptr(st), N.ptr(ws), ws.numel(), N.stream_handle())
    assert int(st.item()) == 0
    k = int(nnz.item())
    co, crow, ccol, sa, sb = (v.cpu().numpy() for v in (co, crow, ccol, sa, sb))
    for r in range(n):
        a = ac[ao[r]:ao[r + 1]]
        b = bc[bo[r]:bo[r + 1]]
        u = np.union1d(a, b)
        got = ccol[co[r]:co[r + 1]]
        assert np.array_equal(got, u)
        assert np.all(crow[co[r]:co[r + 1]] == r)
        for p in range(co[r], co[r + 1]):
            c = ccol[p]
            assert (sa[p] >= 0) == (c in a) and (sb[p] >= 0) == (c in b)
            if sa[p] >= 0:
                assert ac[sa[p]] == c and ao[r] <= sa[p] < ao[r + 1]
            if sb[p] >= 0:
                assert bc[sb[p]] == c and bo[r] <= sb[p] < bo[r + 1]
    assert k == co[n]


def test_autotuner_records_every_candidate(cuda):
    sc = small_scenes()[0]
    s = _solver(sc, torch.float32, "queue")
    s.compute_A()
    (key, times), = s._tuner.timings.items()
    assert len(times) == len(s._tuner.candidates)
    assert s._tuner.best[key] in s._tuner.candidates
    # a second call with the same workload reuses the choice
    s.compute_A()
    assert len(s._tuner.timings) == 1


@pytest.mark.parametrize("cfg", [("separate",), (0, 2, 128, 64), (0, 4, 64, 32), (1, 1, 128, 32), (1, 2, 128, 128)])
def test_every_schedule_assembles_the_same_matrix(cuda, cfg):
    """The per-kind kernels and the persistent work-queue launch (its two
    register variants, with staged tet chunks and class-sorted contact
    chunks) produce the same matrix and force."""
    sc = small_scenes()[2]
    rng = np.random.default_rng(11)
    x = sc.x + rng.normal(scale=0.05 * sc.dhat, size=sc.x.shape)
    out = []
    for assembly in ("generic", "queue"):
        s = _solver(sc, torch.float64, assembly)
        s.states.x.copy_(torch.tensor(x, dtype=torch.float64))
        if assembly == "queue":
            s._static_pattern()
            s._tuner.pick = lambda key, run, reset: cfg
        A = s.compute_A()
        out.append((_dense(A)[0], s.b.cpu().numpy().copy()))
    (Dg, bg), (Dq, bq) = out
    assert np.abs(Dq - Dg).max() <= 1e-12 * np.abs(Dg).max()
    assert np.abs(bq - bg).max() <= 1e-11 * np.abs(bg).max()


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_graph_replayed_compute_A_equals_step_by_step(cuda, dtype):
    """compute_A replayed from its CUDA graph (device-side counts, capacities,
    one host read) assembles the matrix and force of the step-by-step path."""
    sc = small_scenes()[2]
    rng = np.random.default_rng(5)
    x = sc.x + rng.normal(scale=0.05 * sc.dhat, size=sc.x.shape)
    out = []
    for graph in (False, True):
        s = _solver(sc, dtype, "queue")
        s.graph_compute_A = graph
        s.states.x.copy_(torch.tensor(x, dtype=dtype))
        s.compute_A()
        A = s.compute_A()  # with graph: a replay
        assert (getattr(s, "_A_graph", None) is not None) == graph
        assert s.n_contacts + s.n_contacts_pt > 0
        out.append((_dense(A), s.b.double().cpu().numpy().copy(), s.n_contacts, s.n_contacts_pt))
    ((Dg, rg, cg), bg, *ng), ((Dq, rq, cq), bq, *nq) = out
    assert ng == nq
    assert np.array_equal(rg, rq) and np.array_equal(cg, cq)
    tol = 1e-5 if dtype == torch.float32 else 1e-12
    assert np.abs(Dq - Dg).max() <= tol * np.abs(Dg).max()
    assert np.abs(bq - bg).max() <= tol * max(np.abs(bg).max(), 1e-30) * 10
