"""Affine body dynamics kernels and the reduced Newton system against the
CPU oracle oracle/abd.py; the direct reduced assembly against the
reference's triplet pipeline; Newton steps (gpu)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200 import _native as N
from ipc_warp_b200 import scenes
from ipc_warp_b200.abd import AffineBodyDynamics, FixedBVHAffineBodyDynamics
from oracle import abd as oa
from oracle import newton as on

pytestmark = pytest.mark.gpu

DTYPES = [torch.float32, torch.float64]
TOL = {torch.float32: 1e-5, torch.float64: 1e-10}


def _sim(dtype, cls=AffineBodyDynamics, n_side=2, subdiv=1, dhat=0.05, kappa=1e4, gap=5e-3, drop=5e-3, **kw):
    cfg = scenes.abd_balls(n_side=n_side, subdiv=subdiv, gap=gap, drop=drop, seed=3)
    cfg.update(kw)
    return cls(1e-2, density=1000.0, affine_stiffness=1e5, contact_kappa=kappa, dhat=dhat, dtype=dtype, **cfg)


def _host(t):
    return t.double().cpu().numpy()


def _perturb(sim, seed, scale=1e-3):
    rng = np.random.default_rng(seed)
    q = _host(sim.abd_states.q).reshape(-1, 4, 3)
    fixed = _host(sim.abd_fixed).astype(bool)
    d = scale * rng.normal(size=q.shape)
    d[fixed] = 0
    sim.abd_states.q.copy_(torch.tensor((q + d).reshape(-1, 3), dtype=sim.dtype))
    sim._sync_vertices()


def _oracle_args(sim):
    return (_host(sim.abd_states.q).reshape(-1, 4, 3), _host(sim.abd_states.q_tilde).reshape(-1, 4, 3),
            _host(sim.abd_mass).reshape(-1, 4, 4), _host(sim.abd_volume), _host(sim.abd_stiffness),
            sim.abd_fixed.cpu().numpy(), _host(sim.xcs))


def _problem(sim):
    from ipc_warp_b200 import contact

    V = sim.n_nodes
    return on.Problem(xcs=_host(sim.xcs), tets=np.zeros((0, 4), np.int32),
                      edges=sim.soup.edges.cpu().numpy().reshape(-1, 2),
                      triangles=sim.soup.triangles.cpu().numpy().reshape(-1, 3), body=sim.body.cpu().numpy(),
                      mass=np.zeros(V), fixed=np.zeros(V, bool), x_target=np.zeros((V, 3)), material=0, mu=0.0,
                      lam=0.0, dhat=2.0 * contact._thickness, kappa=sim.contact_stiffness, h=sim.h, k_att=0.0,
                      gravity=np.zeros(3), fp64=sim.dtype == torch.float64, exclude_same_body=True)


def _dense(A):
    nnz = int(A.nnz_dev.item())
    off = A.offsets.cpu().numpy()
    cols = A.columns.cpu().numpy()[:nnz]
    vals = _host(A.values[:nnz])
    rows = np.repeat(np.arange(A.nrow), np.diff(off))
    return oa.dense(rows, cols, vals, A.nrow)


@pytest.mark.parametrize("dtype", DTYPES)
def test_vertex_map_predictor_velocity(cuda, dtype):
    sim = _sim(dtype, motors={1: (0.0, 3.0, 0.0)})
    _perturb(sim, 0)
    q, qt, M, vol, stiff, fixed, rest = _oracle_args(sim)
    assert np.allclose(_host(sim.states.x), oa.affine_map(q, rest, sim.body.cpu().numpy()), rtol=0,
                       atol=TOL[dtype] * 10)
    rng = np.random.default_rng(1)
    qd = rng.normal(size=q.shape)
    sim.abd_states.qdot.copy_(torch.tensor(qd.reshape(-1, 3), dtype=dtype))
    sim.abd_states.q0.copy_(sim.abd_states.q)
    sim._prepare_prediction()
    ref = oa.prepare_tilde(q, qd, sim.h, sim.gravity, _host(sim.motor_omega), sim.motor_enabled.cpu().numpy())
    assert np.allclose(_host(sim.abd_states.q_tilde).reshape(-1, 4, 3), ref, atol=TOL[dtype] * 10)
    q1 = q + 1e-3 * rng.normal(size=q.shape)
    sim.abd_states.q.copy_(torch.tensor(q1.reshape(-1, 3), dtype=dtype))
    N.call("ipcb_abd_update_velocity", __import__("ctypes").byref(sim._c_abd), sim.h, N.stream_handle())
    qd_ref, q0_ref = oa.update_velocity(q1, q, sim.h)
    assert np.allclose(_host(sim.abd_states.qdot).reshape(-1, 4, 3), qd_ref, atol=1e-3 if dtype == torch.float32
                       else 1e-9)
    assert np.array_equal(_host(sim.abd_states.q0), _host(sim.abd_states.q))


@pytest.mark.parametrize("dtype", DTYPES)
def test_body_system_and_energy_match_oracle(cuda, dtype):
    sim = _sim(dtype)
    _perturb(sim, 2, scale=3e-2)
    sim.abd_states.q_tilde.copy_(sim.abd_states.q0)
    q, qt, M, vol, stiff, fixed, rest = _oracle_args(sim)
    h2 = sim.h * sim.h
    sim._body_triplets = None
    sim._compute_A_triplets(0, 0)
    bt = sim._body_triplets
    blocks, grad = oa.body_system(q, qt, M, vol, stiff, fixed, h2)
    got = _host(bt.vals).reshape(-1, 4, 4, 3, 3)
    assert np.array_equal(bt.rows.cpu().numpy(), np.repeat(np.arange(4 * len(vol)), 4))
    assert np.abs(got - blocks).max() <= TOL[dtype] * np.abs(blocks).max()
    g = _host(sim.reduced_b).reshape(-1, 4, 3)
    assert np.abs(g - grad).max() <= TOL[dtype] * max(np.abs(grad).max(), 1e-30) * 10
    inertia, ortho = sim._energies()
    ri, ro = oa.body_energy(q, qt, M, vol, stiff, fixed, h2)
    assert abs(inertia - ri) <= 1e-4 * abs(ri) + 1e-12
    assert abs(ortho - ro) <= 1e-4 * abs(ro) + 1e-12


@pytest.mark.parametrize("dtype", DTYPES)
def test_reduced_system_matches_oracle(cuda, dtype):
    sim = _sim(dtype)
    _perturb(sim, 4)
    A = sim.compute_A()
    assert sim.n_contacts + sim.n_contacts_pt > 0
    q, qt, M, vol, stiff, fixed, rest = _oracle_args(sim)
    g_ref, A_ref, n_ee, n_pt = oa.system(_problem(sim), q, qt, M, vol, stiff, fixed, rest, x=_host(sim.states.x))
    assert (n_ee, n_pt) == (sim.n_contacts, sim.n_contacts_pt)
    Ad = _dense(A)
    assert np.abs(Ad - A_ref).max() <= TOL[dtype] * np.abs(A_ref).max() * 10
    g = _host(sim.reduced_b).reshape(-1)
    assert np.abs(g - g_ref.reshape(-1)).max() <= TOL[dtype] * np.abs(g_ref).max() * 10
    # the reference's triplet pipeline gives the same matrix and gradient
    sim.assembly = "triplets"
    B = sim.compute_A()
    assert np.abs(_dense(B) - Ad).max() <= TOL[dtype] * np.abs(Ad).max() * 10
    assert np.abs(_host(sim.reduced_b).reshape(-1) - g).max() <= TOL[dtype] * np.abs(g).max() * 10


def test_fixed_bodies_decouple(cuda):
    sim = _sim(torch.float64)
    _perturb(sim, 5)
    A = _dense(sim.compute_A())
    nb = sim.n_bodies
    f = nb - 1  # the slab
    blk = A[12 * f:12 * f + 12]
    assert np.allclose(blk[:, 12 * f:12 * f + 12], np.eye(12))
    assert np.abs(np.delete(blk, np.s_[12 * f:12 * f + 12], axis=1)).max() == 0
    assert np.abs(_host(sim.reduced_b)[4 * f:4 * f + 4]).max() == 0


@pytest.mark.parametrize("cls", [AffineBodyDynamics, FixedBVHAffineBodyDynamics])
def test_newton_steps_rest_on_ground(cuda, cls):
    sim = _sim(torch.float64, cls=cls)
    for _ in range(3):
        st = sim.step()
        assert st.newton_iterations >= 1
        assert all(a > 0 for a in st.alphas[:-1])
    y = _host(sim.states.x)[sim.body.cpu().numpy() < sim.n_bodies - 1, 1]
    assert y.min() > 0.0  # above the slab top (y = 0)
    e = sim._compute_incremental_energy()
    assert np.isfinite(e)


def test_fixed_bvh_and_dynamic_abd_agree(cuda):
    a = _sim(torch.float64)
    b = _sim(torch.float64, cls=FixedBVHAffineBodyDynamics)
    for _ in range(2):
        a.step()
        b.step()
    qa, qb = _host(a.abd_states.q), _host(b.abd_states.q)
    assert np.abs(qa - qb).max() <= 1e-7 * np.abs(qa).max()


def test_spinning_body_converges_to_stationary_point(cuda):
    v, f = scenes.icosphere(2, 0.5)
    sim = AffineBodyDynamics(5e-3, [(v, f)], gravity=(0, 0, 0), affine_stiffness=1e8, dtype=torch.float64,
                             velocity_tolerance=1e-4)
    sim.set_initial_velocity(0, angular=(1.0, 2.0, 3.0))
    q_prev = _host(sim.abd_states.q).reshape(-1, 4, 3)
    st = sim.step()
    assert st.newton_iterations > 1
    q = _host(sim.abd_states.q).reshape(-1, 4, 3)
    qt = _host(sim.abd_states.q_tilde).reshape(-1, 4, 3)
    M = _host(sim.abd_mass).reshape(-1, 4, 4)
    # the step ends at a stationary point of the incremental potential
    _, grad = oa.body_system(q, qt, M, _host(sim.abd_volume), _host(sim.abd_stiffness), [0], sim.h ** 2)
    scale = np.abs(np.einsum("ij,jk->ik", M[0], q[0] - q_prev[0])).max()
    assert np.abs(grad).max() <= 1e-3 * scale
    # the rotation stays orthogonal under the stiff orthogonality potential
    A = q[0, 1:].T
    assert np.abs(A.T @ A - np.eye(3)).max() < 1e-4
