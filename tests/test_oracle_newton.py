"""The CPU Newton oracle is self-consistent: its gradient and matrix are the
derivatives of its energy, and a step decreases the incremental potential."""
import numpy as np
import pytest

from ipc_warp_b200.newton import lame
from ipc_warp_b200.scenes import two_cubes
from oracle import newton as on


def _problem(material=1, gap=4e-4):
    sc = two_cubes(n=2, gap=gap, angle_deg=15.0, jitter=0.0, seed=0, dhat=1e-3, kappa=1e6)
    mu, lam = lame(1e6, 0.4)
    fixed = sc.xcs[:, 1] <= sc.xcs[:, 1].min() + 1e-9
    p = on.Problem(sc.xcs, sc.tets, sc.edges.reshape(-1, 2), sc.triangles.reshape(-1, 3), sc.body,
                   on.lumped_mass(sc.xcs, sc.tets, 1000.0), fixed, sc.xcs.copy(), material, mu, lam, sc.dhat,
                   sc.kappa, 1e-2, 1e11, np.array([0.0, -9.8, 0.0]), fp64=True)
    return sc, p


@pytest.mark.parametrize("material", [0, 1, 2])
def test_gradient_and_hessian_are_energy_derivatives(material):
    sc, p = _problem(material)
    rng = np.random.default_rng(material)
    x = sc.xcs + rng.normal(scale=2e-5, size=sc.xcs.shape) * ~p.fixed[:, None]
    xt = on.x_tilde(p, sc.xcs, rng.normal(scale=1e-2, size=sc.xcs.shape))
    g, A = on.gradient_hessian(p, x, xt)
    assert len(on._contacts(p, x)[0]) + len(on._contacts(p, x)[1]) > 0
    d = rng.normal(size=x.shape) * ~p.fixed[:, None]
    d /= np.abs(d).max()
    eps = 1e-8
    fd = (on.energy(p, x + eps * d, xt) - on.energy(p, x - eps * d, xt)) / (2 * eps)
    assert abs(fd - float((g * d).sum())) <= 1e-4 * abs(fd) + 1e-9
    # the contact blocks are PSD projections, the rest is the exact Hessian:
    # check the matrix with the barrier switched off
    p.kappa = 0.0
    _, A = on.gradient_hessian(p, x, xt)
    g1, _ = on.gradient_hessian(p, x + eps * d, xt)
    g0, _ = on.gradient_hessian(p, x - eps * d, xt)
    Hd = (g1 - g0).reshape(-1) / (2 * eps)
    Ad = A @ d.reshape(-1)
    assert np.abs(Hd - Ad).max() <= 1e-4 * np.abs(Ad).max()


def test_step_decreases_energy_and_stays_separated():
    sc, p = _problem(gap=2e-3)
    x, xd = sc.xcs.copy(), np.zeros_like(sc.xcs)
    for _ in range(4):
        xt = on.x_tilde(p, x, xd)
        E_start = on.energy(p, x, xt)
        xn, xd, log = on.step(p, x, xd)
        assert on.energy(p, xn, xt) < E_start
        assert np.isfinite(on.energy(p, xn, on.x_tilde(p, xn, xd)))
        assert all(a > 0 for a, _ in log[:-1])
        x = xn
    # the upper cube came down onto the (sagging) top face of the lower one
    assert x[sc.body == 1, 1].min() < sc.xcs[sc.body == 1, 1].min() - 1e-3
