"""Device-side line search (one CUDA graph WHILE loop over the trials) against
the host loop of time_integrator_base.py:514-546 (gpu)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200.newton import FEMContactSolver
from ipc_warp_b200.scenes import two_cubes

pytestmark = pytest.mark.gpu


def _solver(dtype, mode, kappa=1e6):
    sc = two_cubes(n=3, gap=4e-4, angle_deg=15.0, jitter=0.0, seed=0, dhat=1e-3, kappa=kappa)
    fixed = sc.xcs[:, 1] <= sc.xcs[:, 1].min() + 1e-9
    s = FEMContactSolver(sc, material="neo_hookean", E=1e6, nu=0.4, rho=1000.0, h=1e-2, fixed=fixed, dtype=dtype,
                         line_search_mode=mode)
    rng = np.random.default_rng(0)
    x = sc.xcs + rng.normal(scale=2e-5, size=sc.xcs.shape) * ~fixed[:, None]
    s.states.x.copy_(torch.tensor(x, dtype=dtype))
    s.states.x0.copy_(torch.tensor(sc.xcs, dtype=dtype))
    s.states.xdot.copy_(torch.tensor(rng.normal(scale=1e-2, size=x.shape), dtype=dtype))
    return s


def _direction(s):
    s.compute_A()
    s.compute_rhs()
    s.solve()


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_device_search_equals_host(cuda, dtype):
    """Same matrix, direction and state (the direction is not bitwise
    reproducible between solver instances: the force sums use atomics)."""
    s = _solver(dtype, "host")
    _direction(s)
    x0 = s.states.x.clone()
    res = {}
    for mode in ("host", "device"):
        s.line_search_mode = mode
        s.states.x.copy_(x0)
        alpha = s.line_search()
        res[mode] = (alpha, s.stats.energies[-1], s.states.x.double().cpu().numpy().copy())
    (ah, eh, xh), (ad, ed, xd) = res["host"], res["device"]
    assert ah > 0 and ad == ah
    # energies in double: equal up to the summation order of the reductions
    assert ed[0] == pytest.approx(eh[0], rel=1e-12) and ed[1] == pytest.approx(eh[1], rel=1e-12)
    assert np.array_equal(xh, xd)


def test_device_search_backtracks_and_reuses_graph(cuda):
    """A stiff barrier: the search halves from the bound, and a second search
    from the same state replays the captured graph."""
    s = _solver(torch.float64, "device", kappa=1e10)
    _direction(s)
    x0 = s.states.x.clone()
    a1 = s.line_search()
    g1 = s._ls["graph"]
    s.states.x.copy_(x0)
    a2 = s.line_search()
    assert s._ls["graph"] is g1
    s.line_search_mode = "host"
    s.states.x.copy_(x0)
    ah = s.line_search()
    assert a1 == a2 == ah
    assert s.ls_trials >= 1


def test_overflow_falls_back_to_host(cuda):
    s = _solver(torch.float64, "host")
    _direction(s)
    x0 = s.states.x.clone()
    a_ref = s.line_search()
    x_ref = s.states.x.clone()
    s.states.x.copy_(x0)
    s.line_search_mode = "device"
    s.contacts_new.grow(1)  # lists too small for the search: the device loop stops, the host reruns it
    s.contacts_list_new = s.contacts_new
    a = s.line_search()
    assert s.contacts_new.capacity > 1
    assert a == a_ref
    assert torch.equal(s.states.x, x_ref)


def test_newton_steps_with_device_search(cuda):
    """Whole steps with the device search: every accepted trial lowers the
    energy and each step ends by one of the reference's three exits
    (converged, no acceptable step: alpha = 0, or the iteration cap).  This
    scene stalls with tiny steps near contact, and whether a step then ends
    with alpha = 0 or at the cap depends on the rounding of the Hessian sums,
    so the exit is not pinned.  Iterates are not compared with the host
    search step by step: near convergence E1 and E0 agree to rounding, and
    the two sums round differently."""
    s = _solver(torch.float64, "device")
    for _ in range(3):
        st = s.step()
        for a, (e0, e1) in zip(st.alphas, st.energies):
            assert a == 0.0 or e1 < e0
        assert (st.alphas[-1] == 0.0 or st.norms[-1] <= s.vel_tol * s.h
                or st.newton_iterations == s.max_newton)
        assert all(a > 0 for a in st.alphas[:-1])
        assert st.newton_iterations <= s.max_newton
    assert torch.isfinite(s.states.x).all()


def test_newton_iteration_reuses_detection_for_e0(cuda):
    """Inside newton_iteration the device search takes E0's contacts from
    compute_A's detection; E0 and alpha match a search that detects again."""
    s = _solver(torch.float64, "device")
    x0 = s.states.x.clone()
    alpha, _ = s.newton_iteration()
    e0_reused = s.stats.energies[-1][0]
    x1 = s.states.x.clone()
    s.states.x.copy_(x0)
    s.line_search_mode = "device"
    alpha2 = s.line_search()  # direct call: detects at x0 again, same direction
    assert s.stats.energies[-1][0] == pytest.approx(e0_reused, rel=1e-12)
    assert alpha2 == alpha and torch.equal(s.states.x, x1)
