"""Implicit-Euler Newton integrator with contact against the CPU Newton
oracle (time_integrator_base.py:375-546, dynamic_contacts.py:249-308) (gpu)."""
import math

import numpy as np
import pytest
import torch

from ipc_warp_b200.newton import FEMContactSolver, lame, pcg, BlockJacobi
from ipc_warp_b200.scenes import two_cubes
from oracle import newton as on

pytestmark = pytest.mark.gpu

E_YOUNG, NU, RHO, H = 1e6, 0.4, 1000.0, 1e-2


def _scene(gap):
    return two_cubes(n=3, gap=gap, angle_deg=15.0, jitter=0.0, seed=0, dhat=1e-3, kappa=1e6)


def _fixed(sc):
    return sc.xcs[:, 1] <= sc.xcs[:, 1].min() + 1e-9


def _solver(sc, dtype, material="neo_hookean", E=E_YOUNG, **kw):
    return FEMContactSolver(sc, material=material, E=E, nu=NU, rho=RHO, h=H, fixed=_fixed(sc), dtype=dtype, **kw)


def _problem(sc, fp64, material=1, E=E_YOUNG):
    mu, lam = lame(E, NU)
    return on.Problem(sc.xcs, sc.tets, sc.edges.reshape(-1, 2), sc.triangles.reshape(-1, 3), sc.body,
                      on.lumped_mass(sc.xcs, sc.tets, RHO), _fixed(sc),
                      # the attachment targets are the rest positions in the solver's precision
                      sc.xcs.astype(np.float64 if fp64 else np.float32).astype(np.float64), material, mu, lam, sc.dhat,
                      sc.kappa, H, 1e11, np.array([0.0, -9.8, 0.0]), fp64=fp64)


def _state(sc, seed=0):
    """A state in contact: rest positions with small noise (well below the
    gap) and a random velocity."""
    rng = np.random.default_rng(seed)
    x = sc.xcs + rng.normal(scale=2e-5, size=sc.xcs.shape) * ~_fixed(sc)[:, None]
    xdot = rng.normal(scale=1e-2, size=sc.xcs.shape)
    return x, xdot


@pytest.mark.parametrize("fp64", [False, True])
@pytest.mark.parametrize("material", ["snh", "neo_hookean", "stvk"])
def test_gradient_and_matrix_match_oracle(cuda, fp64, material):
    sc = _scene(4e-4)
    dt = torch.float64 if fp64 else torch.float32
    s = _solver(sc, dt, material)
    x, xdot = _state(sc)
    s.states.x.copy_(torch.tensor(x, dtype=dt))
    s.states.x0.copy_(torch.tensor(sc.xcs, dtype=dt))
    s.states.xdot.copy_(torch.tensor(xdot, dtype=dt))
    A = s.compute_A()
    g = s.compute_rhs().double().cpu().numpy()
    assert s.n_contacts + s.n_contacts_pt > 0
    p = _problem(sc, fp64, {"snh": 0, "neo_hookean": 1, "stvk": 2}[material])
    xs = np.asarray(x, dtype=p.dtype)
    xt = on.x_tilde(p, np.asarray(np.asarray(sc.xcs, p.dtype), np.float64), np.asarray(np.asarray(xdot, p.dtype), np.float64))
    g_ref, A_ref = on.gradient_hessian(p, xs, xt)
    tol = 1e-9 if fp64 else 2e-4
    assert np.abs(g - g_ref).max() <= tol * np.abs(g_ref).max()
    rng = np.random.default_rng(1)
    v = rng.normal(size=(len(sc.xcs), 3))
    Av = A.to_scipy() @ v.reshape(-1)
    Av_ref = A_ref @ v.reshape(-1)
    # row-wise backward-error scale |A| |v| (the fixed rows carry h^2 k_att)
    scale = abs(A_ref) @ np.abs(v.reshape(-1))
    assert np.all(np.abs(Av - Av_ref) <= tol * scale)
    # total energy (double) against the oracle's; in single precision the
    # per-tet energy density carries rounding of order mu * eps
    E = s.total_energy()
    E_ref = on.energy(p, xs, xt)
    mu, _ = lame(E_YOUNG, NU)
    atol = 1e-12 if fp64 else H * H * mu * 2.0 * 1e-6
    assert abs(E - E_ref) <= (1e-10 if fp64 else 1e-5) * abs(E_ref) + atol


def test_pcg_direction_matches_direct_solve(cuda):
    sc = _scene(4e-4)
    s = _solver(sc, torch.float64)
    x, xdot = _state(sc, seed=3)
    s.states.x.copy_(torch.tensor(x))
    s.states.x0.copy_(torch.tensor(sc.xcs))
    s.states.xdot.copy_(torch.tensor(xdot))
    s.compute_A()
    s.compute_rhs()
    dx, its, rel = pcg(s.A, s.rhs, BlockJacobi(s.A), tol=1e-11, maxiter=5000)
    assert rel <= 1e-11
    p = _problem(sc, True)
    g_ref, A_ref = on.gradient_hessian(p, x, on.x_tilde(p, sc.xcs, xdot))
    import scipy.sparse.linalg as spla

    ref = spla.spsolve(A_ref.tocsc(), g_ref.reshape(-1)).reshape(-1, 3)
    assert np.abs(dx.cpu().numpy() - ref).max() <= 1e-7 * np.abs(ref).max()


@pytest.mark.parametrize("material", ["snh", "neo_hookean"])
def test_newton_iteration_matches_oracle(cuda, material):
    """One Newton iteration in double (matrix, tight PCG solve, CCD bound,
    backtracking) lands on the oracle's iterate."""
    sc = _scene(4e-4)
    m = {"snh": 0, "neo_hookean": 1}[material]
    s = _solver(sc, torch.float64, material, tol=1e-11, maxiter=5000)
    x, xdot = _state(sc, seed=5)
    s.states.x.copy_(torch.tensor(x))
    s.states.x0.copy_(torch.tensor(sc.xcs))
    s.states.xdot.copy_(torch.tensor(xdot))
    alpha, norm = s.newton_iteration()
    p = _problem(sc, True, m)
    xt = on.x_tilde(p, sc.xcs, xdot)
    g, A = on.gradient_hessian(p, x, xt)
    import scipy.sparse.linalg as spla

    dx = spla.spsolve(A.tocsc(), g.reshape(-1)).reshape(-1, 3)
    xr, alpha_r, E0, E1 = on.line_search(p, x, dx, xt)
    assert alpha_r > 0
    assert abs(alpha - alpha_r) <= 2e-6 * alpha_r
    assert abs(norm - np.abs(dx).max()) <= 1e-7 * norm
    assert np.abs(s.states.x.cpu().numpy() - xr).max() <= 1e-8
    assert abs(s.stats.energies[-1][0] - E0) <= 1e-10 * abs(E0)


def _falling_scene():
    """The upper cube, tilted so that a corner comes down first, falls at
    0.1 m/s onto the lower one, whose bottom layer is fixed."""
    return two_cubes(n=3, gap=2e-3, angle_deg=15.0, tilt_deg=7.0, jitter=0.0, seed=0, dhat=1e-3, kappa=1e11)


@pytest.mark.parametrize("fp64", [False, True])
def test_falling_cube_trajectory(cuda, fp64):
    """Every accepted line search lowers the total energy, the contact set is
    never crossed (finite barrier energy at every frame) and, in double, the
    frames follow the CPU Newton oracle."""
    sc = _falling_scene()
    dt = torch.float64 if fp64 else torch.float32
    E = 1e7
    vel_tol = 1e-4 if fp64 else 5e-2
    s = _solver(sc, dt, E=E, vel_tol=vel_tol, tol=1e-10 if fp64 else 1e-4, maxiter=2000 if fp64 else 200)
    v0 = np.zeros_like(sc.xcs)
    v0[sc.body == 1, 1] = -0.1
    s.states.xdot.copy_(torch.tensor(v0, dtype=dt))
    p = _problem(sc, fp64, E=E)
    xr, xdr = sc.xcs.copy(), v0.copy()
    had_contact = False
    for frame in range(8):
        st = s.step()
        assert st.newton_iterations < s.max_newton
        for (E0, E1), a in zip(st.energies, st.alphas):
            if a > 0:
                assert E1 < E0
        x = s.states.x.double().cpu().numpy()
        Ef = on.energy(p, x.astype(p.dtype), on.x_tilde(p, x, np.zeros_like(x)))
        assert math.isfinite(Ef)
        had_contact |= (s.n_contacts + s.n_contacts_pt) > 0
        if fp64:
            xr, xdr, _ = on.step(p, xr, xdr, vel_tol=vel_tol)
            assert np.abs(x - xr).max() <= 1e-5, frame
    assert had_contact
    # the corner came down onto the lower cube (separation is the finite
    # barrier energy above)
    assert x[sc.body == 1, 1].min() < sc.xcs[sc.body == 1, 1].min() - 1e-3


def test_direct_solver_step_matches_pcg_step(cuda):
    """The reference's direct path (solve_ldlt) and PCG give the same Newton
    iterate; a PCG capped at one iteration falls back to the direct solve."""
    sc = _scene(4e-4)
    x, xdot = _state(sc, seed=9)
    out = {}
    for name, kw in (("direct", dict(linear_solver="direct")), ("pcg", dict(tol=1e-11, maxiter=5000)),
                     ("fallback", dict(tol=1e-11, maxiter=1))):
        s = _solver(sc, torch.float64, **kw)
        s.states.x.copy_(torch.tensor(x))
        s.states.x0.copy_(torch.tensor(sc.xcs))
        s.states.xdot.copy_(torch.tensor(xdot))
        s.newton_iteration()
        out[name] = (s.states.x.cpu().numpy(), s.stats.fallbacks)
    assert np.abs(out["direct"][0] - out["pcg"][0]).max() <= 1e-9
    assert np.abs(out["direct"][0] - out["fallback"][0]).max() <= 1e-12
    assert out["fallback"][1] == 1 and out["pcg"][1] == 0
