"""What the trained preconditioner gains over the method without it: PCG
iterations at relative residual 1e-6 on Newton systems from scenes and seeds
the training did not see, with the direct solve as judge (gpu)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200 import learned as L
from ipc_warp_b200 import train_preconditioner as T
from ipc_warp_b200.bsr import bsr_mv
from ipc_warp_b200.direct import DirectSolver
from ipc_warp_b200.newton import BlockJacobi, pcg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems(cuda):
    return (T.cube_systems(3, 11, 8) + T.rod_systems(4, 12, 8)
            + T.rod_systems(4, 13, 8, side=3, cells=(4, 4, 32), gap_over_dhat=0.5))


def test_learned_pcg_needs_fewer_iterations(cuda, systems):
    net = L.Net.load(L.DEFAULT_WEIGHTS, device=cuda)
    its_j, its_l = 0, 0
    for A in systems:
        g = torch.Generator(device=cuda).manual_seed(A.nrow)
        b = torch.randn((A.nrow, 3), generator=g, device=cuda, dtype=A.dtype)
        _, ij, rj = pcg(A, b, BlockJacobi(A), 1e-6, 20000)
        x, il, rl = pcg(A, b, L.LearnedPreconditioner(net)(A), 1e-6, 20000)
        assert rj <= 1e-6 and rl <= 1e-6
        # true residual of the learned solve
        res = b - bsr_mv(A, x)
        # float32 SpMV of a stiff system: the true residual carries |A||x| eps
        assert float(res.double().norm() / b.double().norm()) <= 1e-4
        its_j += ij
        its_l += il
    assert its_l <= 0.75 * its_j, (its_l, its_j)


def test_learned_pcg_agrees_with_direct_solve(cuda, systems):
    net = L.Net.load(L.DEFAULT_WEIGHTS, device=cuda)
    A = systems[-1]
    b = torch.randn((A.nrow, 3), device=cuda, dtype=A.dtype)
    x, its, rel = pcg(A, b, L.LearnedPreconditioner(net)(A), 1e-6, 20000)
    xd = DirectSolver("metis")(A, b)
    assert float((x - xd).double().norm() / xd.double().norm()) <= 1e-3


@pytest.mark.parametrize("kind", ["jacobi", "learned"])
@pytest.mark.parametrize("use_graph", [False, True])
def test_device_pcg_matches_host_pcg(cuda, systems, kind, use_graph):
    """The device-resident PCG (batched, graph-replayed) reaches the same
    residual in the same number of iterations as the host-driven loop."""
    from ipc_warp_b200.newton import DevicePcg, JacobiPrecond

    net = L.Net.load(L.DEFAULT_WEIGHTS, device=cuda)
    dp = DevicePcg(batch=8, use_graph=use_graph)
    for A in systems[::3]:
        b = torch.randn((A.nrow, 3), device=cuda, dtype=A.dtype)
        if kind == "jacobi":
            xh, ih, rh = pcg(A, b, BlockJacobi(A), 1e-6, 20000)
            M = JacobiPrecond(A)
        else:
            # the device apply uses the bf16 mirror of the factor
            M = L.LearnedFactor(net, A)
            xh, ih, rh = pcg(A, b, L.LearnedPreconditioner(net)(A), 1e-6, 20000)
        x, it, rel, status = dp.solve(A, b, M, 1e-6, 20000)
        assert status == 0 and rel <= 1e-6
        res = b - bsr_mv(A, x)
        # float32 SpMV of a stiff system: the true residual carries |A||x| eps
        assert float(res.double().norm() / b.double().norm()) <= 1e-4
        assert abs(it - ih) <= max(3, 0.1 * ih), (it, ih)
