"""A CCD query that runs out of its traversal stack, its visit bound or its
root iterations (IPCB_STATUS_STACK / IPCB_STATUS_ROOT_ITERS) may have missed
an impact, so its TOI is no bound: every consumer of the TOI must refuse the
step (alpha = 0) and count the refusal (gpu).

The failing query is faked on the host: the status word the kernels would
have written is set after the real CCD launches, the way a failed call is
faked in tests (no kernel is made to fail)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200 import contact
from ipc_warp_b200.newton import FEMContactSolver
from ipc_warp_b200.pipeline import ContactPipeline
from ipc_warp_b200.scenes import two_cubes

pytestmark = pytest.mark.gpu


def _scene():
    return two_cubes(n=3, gap=4e-4, angle_deg=15.0, jitter=0.0, seed=0, dhat=1e-3, kappa=1e6)


class _FailingCcd:
    """Mixin: after the real CCD launches, the status word says a query ran
    out of its bound (bit 1 = stack / visits, bit 2 = root iterations)."""
    fail_bits = contact.QUERY_FAILED & 1

    def _launch_ccd(self, dx, reset_status=True):
        super()._launch_ccd(dx, reset_status)
        self._status.fill_(self.fail_bits)

    def _ccd_launches(self, dx):
        super()._ccd_launches(dx)
        self._status.fill_(self.fail_bits)


class FailingSolver(_FailingCcd, FEMContactSolver):
    pass


class FailingPipeline(_FailingCcd, ContactPipeline):
    def _copy_results(self, e):
        self._status.fill_(self.fail_bits)
        super()._copy_results(e)


def _solver(cls, mode, bits):
    sc = _scene()
    fixed = sc.xcs[:, 1] <= sc.xcs[:, 1].min() + 1e-9
    s = cls(sc, material="neo_hookean", E=1e6, nu=0.4, rho=1000.0, h=1e-2, fixed=fixed, dtype=torch.float64,
            line_search_mode=mode)
    s.fail_bits = bits
    rng = np.random.default_rng(0)
    x = sc.xcs + rng.normal(scale=2e-5, size=sc.xcs.shape) * ~fixed[:, None]
    s.states.x.copy_(torch.tensor(x, dtype=torch.float64))
    s.states.x0.copy_(torch.tensor(sc.xcs, dtype=torch.float64))
    s.states.xdot.copy_(torch.tensor(rng.normal(scale=1e-2, size=x.shape), dtype=torch.float64))
    return s


@pytest.mark.parametrize("mode", ["host", "device"])
@pytest.mark.parametrize("bits", [1, 2])
def test_newton_line_search_refuses_a_failed_ccd(cuda, mode, bits):
    s = _solver(FailingSolver, mode, bits)
    x0 = s.states.x.clone()
    alpha, norm = s.newton_iteration()
    assert alpha == 0.0 and norm == 0.0
    assert s.stats.ccd_refusals == 1
    assert torch.equal(s.states.x, x0)
    # the same state with a query that did not fail takes a step
    ok = _solver(FEMContactSolver, mode, 0)
    a_ok, _ = ok.newton_iteration()
    assert a_ok > 0.0 and ok.stats.ccd_refusals == 0


def test_collision_free_step_refuses_a_failed_ccd(cuda):
    sc = _scene()
    pipe = FailingPipeline.from_scene(sc, dtype=torch.float32, device=cuda)
    dx = torch.zeros_like(pipe.states.x)
    dx[:, 1] = 1e-4
    assert pipe.collision_free_step(dx) == 0.0
    assert pipe.ccd_refusals == 1 and pipe.query_status & 1
    good = ContactPipeline.from_scene(sc, dtype=torch.float32, device=cuda)
    assert good.collision_free_step(dx) > 0.0 and good.ccd_refusals == 0


@pytest.mark.parametrize("use_graph", [False, True])
def test_pipeline_iteration_refuses_a_failed_query(cuda, use_graph):
    sc = _scene()
    pipe = FailingPipeline.from_scene(sc, dtype=torch.float32, device=cuda)
    pipe.use_graph = use_graph
    dx = torch.zeros_like(pipe.states.x)
    dx[:, 1] = 1e-4
    for _ in range(3):  # eager pass, capture, replay
        r = pipe.iteration(dx)
        assert r.alpha == 0.0 and r.status & 1
    good = ContactPipeline.from_scene(sc, dtype=torch.float32, device=cuda)
    r = good.iteration(dx)
    assert r.alpha > 0.0 and r.status == 0
