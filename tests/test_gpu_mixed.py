"""Mixed FEM + affine-body Newton system (ipc_warp_b200.mixed, csrc/mixed.cu)
against the CPU oracle oracle/mixed.py, and short trajectories of the
wrecking-balls configuration that must stay intersection-free (gpu)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200 import contact, scenes
from ipc_warp_b200.mixed import MixedSolver
from oracle import mixed as om
from oracle import newton as on

pytestmark = pytest.mark.gpu

DTYPES = [torch.float32, torch.float64]
TOL = {torch.float32: 1e-5, torch.float64: 1e-10}


def _host(t):
    return t.double().cpu().numpy()


def _oracle(s: MixedSolver):
    V = s.n_verts
    p = on.Problem(xcs=_host(s.soup.xcs), tets=s.tets.cpu().numpy(), edges=s.soup.edges.cpu().numpy().reshape(-1, 2),
                   triangles=s.soup.triangles.cpu().numpy().reshape(-1, 3), body=s.soup.body.cpu().numpy(),
                   mass=np.zeros(V), fixed=np.zeros(V, bool), x_target=np.zeros((V, 3)), material=s.material,
                   mu=s.mu, lam=s.lam, dhat=2.0 * contact._thickness, kappa=s.contact_stiffness, h=s.h, k_att=0.0,
                   gravity=np.zeros(3), fp64=s.dtype == torch.float64, exclude_same_body=s.disable_self_collision)
    m = om.Mixed(n_fem=s.n_fem, body=s.body_local.cpu().numpy(), fixed=s.abd_fixed.cpu().numpy(),
                 rest=_host(s.soup.xcs), fem_mass=_host(s.fem_mass), M=_host(s.abd_mass).reshape(-1, 4, 4),
                 volume=_host(s.abd_volume), stiffness=_host(s.abd_stiffness), pin_rest=_host(s.pin_rest),
                 pin_target=_host(s.pin_target), pin_k=_host(s.pin_k))
    return p, m


def _solver(dtype, assembly="queue", affine_stiffness=1e5, **kw):
    sc = scenes.mixed_touching(**kw)
    return MixedSolver(sc, E=1e5, nu=0.4, h=1e-2, dtype=dtype, affine_stiffness=affine_stiffness, maxiter=2000,
                       assembly=assembly)


def _perturb(s: MixedSolver, seed, scale=2e-5):
    rng = np.random.default_rng(seed)
    q = _host(s.q)
    d = scale * rng.normal(size=q.shape)
    fixed = _host(s.abd_fixed).astype(bool)
    for b in np.flatnonzero(fixed):
        o = s.n_fem + 4 * b
        d[o:o + 4] = 0
    s.q.copy_(torch.tensor(q + d, dtype=s.dtype))
    s._sync()


@pytest.mark.parametrize("dtype", DTYPES)
def test_mixed_system_matches_oracle(cuda, dtype):
    s = _solver(dtype)
    _perturb(s, 1)
    A = s.compute_A()
    n_ee, n_pt = s.n_contacts, s.n_contacts_pt
    assert n_ee + n_pt > 0
    p, m = _oracle(s)
    g_ref, A_ref, ne, npt = om.system(p, m, _host(s.q), _host(s.xt_f), _host(s.qt_a), x=_host(s.x))
    assert (ne, npt) == (n_ee, n_pt)
    # every body pair of the scene is in contact: ball-ball, ball-cube, ball-ground, cube-ground
    body = s.soup.body.cpu().numpy()
    recs = np.concatenate([s.contacts_new.records(n_ee)[:, :4].cpu().numpy(),
                           s.contacts_pt.records(n_pt)[:, :4].cpu().numpy()])
    pairs = {tuple(sorted(set(body[r].tolist()))) for r in recs}
    assert {(1, 2), (0, 1), (1, 3), (2, 3), (0, 3)} <= pairs, pairs
    Ad = A.to_scipy().toarray()
    Ar = A_ref.toarray()
    assert np.abs(Ad - Ar).max() <= TOL[dtype] * np.abs(Ar).max() * 10
    g = _host(s.rhs)
    assert np.abs(g - g_ref).max() <= TOL[dtype] * np.abs(g_ref).max() * 10
    # the matrix is symmetric and its coupling blocks between the cube's
    # unknowns and ball 0's are non-zero
    assert np.abs(Ad - Ad.T).max() <= TOL[dtype] * np.abs(Ad).max() * 10
    o = 3 * s.n_fem
    assert np.abs(Ad[:o, o:o + 12]).max() > 0


@pytest.mark.parametrize("cfg", [(0, 2, 128, 64), (1, 1, 128, 32), (0, 4, 64, 32)])
def test_fused_terms_equal_per_kind_kernels(cuda, cfg):
    """The persistent launch over contact records, tets and affine-body items
    assembles the same matrix and gradient as the per-kind kernels."""
    out = []
    for assembly in ("separate", "queue"):
        s = _solver(torch.float64, assembly=assembly)
        _perturb(s, 3)
        if assembly == "queue":
            s._tuner.pick = lambda key, run, reset: cfg
        A = s.compute_A()
        assert s.n_contacts + s.n_contacts_pt > 0
        out.append((A.to_scipy().toarray(), _host(s.rhs)))
    (A0, g0), (A1, g1) = out
    assert np.abs(A1 - A0).max() <= 1e-12 * np.abs(A0).max()
    assert np.abs(g1 - g0).max() <= 1e-11 * np.abs(g0).max()


@pytest.mark.parametrize("dtype", DTYPES)
def test_mixed_energy_matches_oracle(cuda, dtype):
    s = _solver(dtype)
    _perturb(s, 2)
    e = s.total_energy()
    p, m = _oracle(s)
    ref = om.energy(p, m, _host(s.q), _host(s.xt_f), _host(s.qt_a), x=_host(s.x))
    # float32: the body inertia and orthogonality sums run in float (as
    # test_gpu_abd's energies), so the bound is theirs
    assert abs(e - ref) <= (1e-4 if dtype == torch.float32 else 1e-10) * abs(ref) + 1e-12


def test_mixed_newton_steps_rest(cuda):
    """The touching scene under gravity: Newton converges every step, no
    surface crossing, the pinned ball stays rigid, the ground does not move."""
    s = _solver(torch.float64, affine_stiffness=1e8)
    q0 = _host(s.q)
    ground = s.n_fem + 4 * 2
    for k in range(5):
        st = s.step()
        assert st.newton_iterations < s.max_newton, k
        assert st.ccd_refusals == 0
        assert s.edge_triangle_crossings()[0] == 0, k
    q = _host(s.q)
    assert np.isfinite(q).all()
    assert np.abs(q[ground:ground + 4] - q0[ground:ground + 4]).max() == 0.0
    assert s.orthogonality_error() < 1e-3


def test_wrecking_balls_trajectory(cuda):
    """Four balls of the wrecking-balls configuration, released at seeded
    angles, strike their cube stacks: every step converges, no surface
    crossing, the balls stay rigid, the ground stays put, and the balls
    end up touching the cubes (affine-FEM contact records)."""
    sc = scenes.wrecking_balls(n_balls=4, subdiv=3, cube_cells=3, ground_quads=16, max_angle_deg=60.0,
                               kappa=1e12, seed=2)
    s = MixedSolver(sc, E=5e5, nu=0.4, h=1e-2, dtype=torch.float32, maxiter=2000)
    q0 = _host(s.q)
    n_fem_bodies = int(sc.fem.body.max()) + 1
    body = s.soup.body.cpu().numpy()
    hit = False
    for k in range(60):
        st = s.step()
        assert st.newton_iterations < s.max_newton, k
        assert st.ccd_refusals == 0, k
        assert s.edge_triangle_crossings()[0] == 0, k
        n_ee, n_pt = s.n_contacts, s.n_contacts_pt
        recs = np.concatenate([s.contacts_new.records(n_ee)[:, :4].cpu().numpy(),
                               s.contacts_pt.records(n_pt)[:, :4].cpu().numpy()])
        b = body[recs]
        ball = ((b >= n_fem_bodies) & (b < n_fem_bodies + 4)).any(axis=1)
        hit |= bool((ball & (b < n_fem_bodies).any(axis=1)).any())
    q = _host(s.q)
    assert np.isfinite(q).all()
    g = s.n_fem + 4 * (len(sc.bodies) - 1)
    assert np.abs(q[g:g + 4] - q0[g:g + 4]).max() == 0.0
    assert s.orthogonality_error() < 1e-3
    assert hit


def test_mixed_system_matches_oracle_at_impact(cuda):
    """The Newton matrix and gradient of the 4-ball wrecking-balls scene in
    float64, taken at the first step where a ball touches its cubes, against
    the oracle's J^T H J assembly (sparse comparison)."""
    sc = scenes.wrecking_balls(n_balls=4, subdiv=3, cube_cells=3, ground_quads=16, max_angle_deg=60.0,
                               kappa=1e12, seed=2)
    s = MixedSolver(sc, E=5e5, nu=0.4, h=1e-2, dtype=torch.float64, maxiter=4000)
    n_fem_bodies = int(sc.fem.body.max()) + 1
    body = s.soup.body.cpu().numpy()
    for k in range(80):
        s.step()
        s.prepare()
        s.compute_A()
        n_ee, n_pt = s.n_contacts, s.n_contacts_pt
        recs = np.concatenate([s.contacts_new.records(n_ee)[:, :4].cpu().numpy(),
                               s.contacts_pt.records(n_pt)[:, :4].cpu().numpy()])
        b = body[recs]
        ball = ((b >= n_fem_bodies) & (b < n_fem_bodies + 4)).any(axis=1)
        if bool((ball & (b < n_fem_bodies).any(axis=1)).any()):
            break
    else:
        pytest.fail("no ball reached its cubes")
    p, m = _oracle(s)
    g_ref, A_ref, ne, npt = om.system(p, m, _host(s.q), _host(s.xt_f), _host(s.qt_a), x=_host(s.x))
    assert (ne, npt) == (s.n_contacts, s.n_contacts_pt)
    d = (s.A.to_scipy().tocsr() - A_ref).tocoo()
    scale = abs(A_ref).max()
    assert (abs(d.data).max() if d.nnz else 0.0) <= 1e-9 * scale
    g = _host(s.rhs)
    assert np.abs(g - g_ref).max() <= 1e-9 * np.abs(g_ref).max()


@pytest.mark.parametrize("dtype", DTYPES)
def test_body_block_preconditioner(cuda, dtype):
    """The 12x12 body blocks (ipcb_group_jacobi) invert the matrix's diagonal
    body blocks, and the PCG preconditioned by them (3x3 blocks for the FEM
    rows) reaches the direct solution in no more iterations than plain 3x3
    block Jacobi."""
    import scipy.sparse.linalg as sla

    from ipc_warp_b200.newton import DevicePcg, JacobiPrecond

    s = _solver(torch.float64)
    _perturb(s, 4)
    A64 = s.compute_A()
    Ad = A64.to_scipy().toarray()
    ref = sla.spsolve(A64.to_scipy().tocsc(), _host(s.rhs).ravel())
    if dtype == torch.float32:
        s = _solver(dtype)
        _perturb(s, 4)
        s.compute_A()
    A = s.A
    M = JacobiPrecond(A, groups=(s.n_fem, s.n_bodies))
    Dg = M.dinv_group.double().cpu().numpy()
    o = 3 * s.n_fem
    for g in range(s.n_bodies):
        blk = Ad[o + 12 * g:o + 12 * g + 12, o + 12 * g:o + 12 * g + 12]
        err = np.abs(Dg[g] @ blk - np.eye(12)).max()
        assert err <= (1e-3 if dtype == torch.float32 else 1e-9), (g, err)
    its = {}
    for name, groups in (("body_block", (s.n_fem, s.n_bodies)), ("jacobi", None)):
        pcg = DevicePcg()
        M = JacobiPrecond(A, groups=groups)
        x, it, rel, status = pcg.solve(A, s.rhs, M, 1e-8 if dtype == torch.float64 else 1e-5, 4000)
        assert status == 0 and rel <= (1e-8 if dtype == torch.float64 else 1e-5), (name, rel, status)
        xr = _host(x).ravel()
        assert np.abs(xr - ref).max() <= (1e-5 if dtype == torch.float64 else 1e-2) * np.abs(ref).max(), name
        its[name] = it
    assert its["body_block"] <= its["jacobi"], its


def test_body_block_groups_must_cover_rows(cuda):
    from ipc_warp_b200.newton import JacobiPrecond

    s = _solver(torch.float64)
    s.compute_A()
    with pytest.raises(ValueError):
        JacobiPrecond(s.A, groups=(s.n_fem + 1, s.n_bodies))


@pytest.mark.parametrize("fp64", [False, True])
def test_group_jacobi_random_and_singular_blocks(cuda, fp64):
    """ipcb_group_jacobi on a small block matrix: 2 point rows and 3 groups of
    4 block rows; groups 0 and 2 get random SPD 12x12 blocks (their inverse
    is returned), group 1 an all-zero block (singular: the identity is
    returned and IPCB_STATUS_PATTERN is raised)."""
    from ipc_warp_b200 import _native as N
    from ipc_warp_b200.bsr import bsr_from_triplets

    dtype = torch.float64 if fp64 else torch.float32
    n_point, n_groups = 2, 3
    nrow = n_point + 4 * n_groups
    rng = np.random.default_rng(7)
    dense = np.zeros((3 * nrow, 3 * nrow))
    for i in range(n_point):
        dense[3 * i:3 * i + 3, 3 * i:3 * i + 3] = np.eye(3) * (2.0 + i)
    for g in (0, 2):
        m = rng.normal(size=(12, 12))
        o = 3 * n_point + 12 * g
        dense[o:o + 12, o:o + 12] = m @ m.T + 12 * np.eye(12)
    rows, cols, vals = [], [], []
    for bi in range(nrow):
        for bj in range(nrow):
            blk = dense[3 * bi:3 * bi + 3, 3 * bj:3 * bj + 3]
            if np.any(blk) or bi == bj:
                rows.append(bi)
                cols.append(bj)
                vals.append(blk)
    A = bsr_from_triplets(nrow, nrow, torch.tensor(rows, dtype=torch.int32, device=cuda),
                          torch.tensor(cols, dtype=torch.int32, device=cuda),
                          torch.tensor(np.array(vals), dtype=dtype, device=cuda))
    out = torch.empty((n_groups, 12, 12), dtype=dtype, device=cuda)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    N.call("ipcb_group_jacobi", n_point, n_groups, N.ptr(A.offsets), N.ptr(A.columns), N.ptr(A.values), int(fp64),
           N.ptr(out), N.ptr(status), N.stream_handle())
    got = out.double().cpu().numpy()
    assert int(status.item()) & 16
    assert np.array_equal(got[1], np.eye(12))
    for g in (0, 2):
        o = 3 * n_point + 12 * g
        ref = np.linalg.inv(dense[o:o + 12, o:o + 12])
        assert np.abs(got[g] - ref).max() <= (1e-12 if fp64 else 1e-6) * np.abs(ref).max()
    # bad arguments are refused before any launch
    with pytest.raises(N.NativeError):
        N.call("ipcb_group_jacobi", -1, n_groups, N.ptr(A.offsets), N.ptr(A.columns), N.ptr(A.values), int(fp64),
               N.ptr(out), N.ptr(status), N.stream_handle())


def test_pcg_initial_guess(cuda):
    """DevicePcg from an initial guess (ipcb_pcg.x0): the same solution to the
    tolerance, fewer iterations from a close guess, and zero for b = 0."""
    import scipy.sparse.linalg as sla

    from ipc_warp_b200.newton import DevicePcg, JacobiPrecond

    s = _solver(torch.float64)
    _perturb(s, 5)
    A = s.compute_A()
    ref = sla.spsolve(A.to_scipy().tocsc(), _host(s.rhs).ravel())
    M = JacobiPrecond(A, groups=(s.n_fem, s.n_bodies))
    pcg = DevicePcg()
    x, it0, rel, status = pcg.solve(A, s.rhs, M, 1e-8, 4000)
    assert status == 0 and rel <= 1e-8
    guess = torch.tensor(0.9 * ref.reshape(-1, 3), dtype=torch.float64, device=cuda)
    x, it1, rel, status = pcg.solve(A, s.rhs, M, 1e-8, 4000, x0=guess)
    assert status == 0 and rel <= 1e-8
    assert np.abs(_host(x).ravel() - ref).max() <= 1e-5 * np.abs(ref).max()
    assert it1 < it0, (it1, it0)
    x, _, _, status = pcg.solve(A, torch.zeros_like(s.rhs), M, 1e-8, 4000, x0=guess)
    assert status == 0 and not bool(x.any())


@pytest.mark.parametrize("dtype", DTYPES)
def test_device_line_search_matches_host(cuda, dtype):
    """The mixed solver's line search on the device (trials in one WHILE-graph
    launch) against the host loop from the same state and direction: the
    same step and energies (to rounding), and the same q after it."""
    out = []
    for mode in ("host", "device"):
        s = _solver(dtype)
        s.line_search_mode = mode
        _perturb(s, 8)
        s.prepare()
        s.compute_A()
        s.solve()
        alpha = s.line_search()
        E0, E1 = s.stats.energies[-1]
        out.append((alpha, E0, E1, _host(s.q)))
    (ah, e0h, e1h, qh), (ad, e0d, e1d, qd) = out
    tol = 1e-9 if dtype == torch.float64 else 1e-4
    assert 0.0 < ah <= 1.0 and ad == pytest.approx(ah, rel=1e-12)
    assert e0d == pytest.approx(e0h, rel=tol) and e1d == pytest.approx(e1h, rel=tol)
    assert e1d < e0d
    assert np.abs(qd - qh).max() <= (1e-12 if dtype == torch.float64 else 1e-5) * max(np.abs(qh).max(), 1.0)


def test_device_line_search_steps_rest(cuda):
    """A few steps of the touching scene with the device search: converged,
    intersection-free, the ground does not move (as with the host search)."""
    s = _solver(torch.float64, affine_stiffness=1e8)
    assert s.line_search_mode == "device"
    q0 = _host(s.q)
    ground = s.n_fem + 4 * 2
    for k in range(5):
        st = s.step()
        assert st.newton_iterations < s.max_newton, k
        assert st.ccd_refusals == 0
        assert s.edge_triangle_crossings()[0] == 0, k
    q = _host(s.q)
    assert np.abs(q[ground:ground + 4] - q0[ground:ground + 4]).max() == 0.0


@pytest.mark.parametrize("dtype", DTYPES)
def test_fixed_pattern_assembly_equals_sorted_assembly(cuda, dtype):
    """A as the union of the fixed pattern (gathered FEM mass, tet, body and
    pin blocks) and the reduced contact BSR equals the sort-based assembly
    of all triplets, over two Newton iterations (the second reuses the slot
    map)."""
    mats = []
    for fixed in (True, False):
        s = _solver(dtype)
        s.fixed_pattern = fixed
        _perturb(s, 9)
        s.prepare()
        out = []
        for it in range(2):
            A = s.compute_A()
            assert s.n_contacts + s.n_contacts_pt > 0
            out.append(A.to_scipy().toarray())
            if it == 0:
                s.solve()
                s.line_search()
        mats.append(out)
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    for a, b in zip(*mats):
        assert np.abs(a - b).max() <= tol * np.abs(b).max()
