"""ContactPipeline.iteration (counts on the device, one host read at the
end) against the same iteration through the public calls one stage at a
time (gpu)."""
import numpy as np
import pytest
import torch

from helpers import small_scenes
from ipc_warp_b200.pipeline import ContactPipeline

pytestmark = pytest.mark.gpu


def _pipe(sc, dtype, cuda, seed=2):
    pipe = ContactPipeline.from_scene(sc, dtype=dtype, device=cuda)
    rng = np.random.default_rng(seed)
    dx = torch.tensor(rng.normal(scale=0.3 * sc.dhat, size=sc.x.shape), dtype=dtype, device=cuda)
    return pipe, dx


def _bsr(pipe):
    H = pipe.collision_hessian
    nnz = H.nnz_sync()
    return H.offsets.clone(), H.columns[:nnz].clone(), H.values[:nnz].double().clone()


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_iteration_equals_stepwise(cuda, idx, dtype):
    sc = small_scenes()[idx]
    pipe, dx = _pipe(sc, dtype, cuda)
    r1 = pipe.iteration(dx)
    o1, c1, v1 = _bsr(pipe)
    b1 = pipe.b.double().clone()
    r2 = pipe.iteration_stepwise()
    o2, c2, v2 = _bsr(pipe)
    b2 = pipe.b.double().clone()
    assert (r1.n_ee, r1.n_pt) == (r2.n_ee, r2.n_pt) and r1.n_ee + r1.n_pt > 0
    assert r1.alpha == r2.alpha  # TOI by atomicMin: exact
    assert r1.energy == pytest.approx(r2.energy, rel=1e-12)
    # list order (DCD atomics) and force atomics differ between runs: values to rounding
    assert torch.equal(o1, o2) and torch.equal(c1, c2)
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    scale = v2.abs().amax(dim=(1, 2), keepdim=True).clamp_min(1e-300)
    assert ((v1 - v2).abs() <= tol * scale).all()
    assert (b1 - b2).abs().max() <= tol * max(b2.abs().max().item(), 1e-300)


def test_overflowed_list_falls_back(cuda):
    sc = small_scenes()[2]
    pipe, dx = _pipe(sc, torch.float32, cuda)
    ref = pipe.iteration(dx)
    pipe.contacts_new.grow(1)  # too small: the device-count pass overflows, the stepwise pass regrows
    pipe.contacts_list_new = pipe.contacts_new
    r = pipe.iteration(dx)
    assert pipe.contacts_new.capacity >= r.n_ee > 1
    assert (r.n_ee, r.n_pt, r.alpha) == (ref.n_ee, ref.n_pt, ref.alpha)
    assert r.energy == pytest.approx(ref.energy, rel=1e-12)


def test_graph_replay_equals_stepwise(cuda):
    """Eager pass, then capture, then replays with a new direction each time."""
    sc = small_scenes()[3]
    pipe, dx = _pipe(sc, torch.float32, cuda)
    for k in range(4):
        dxk = dx * (1.0 + 0.25 * k)
        r = pipe.iteration(dxk)
        o, c, v = _bsr(pipe)
        ref = pipe.iteration_stepwise()
        o2, c2, v2 = _bsr(pipe)
        assert (r.n_ee, r.n_pt, r.alpha) == (ref.n_ee, ref.n_pt, ref.alpha)
        assert r.energy == pytest.approx(ref.energy, rel=1e-12)
        assert torch.equal(o, o2) and torch.equal(c, c2)
        assert ((v - v2).abs() <= 1e-5 * v2.abs().amax(dim=(1, 2), keepdim=True).clamp_min(1e-30)).all()
    assert pipe._graph is not None  # the later calls replayed it, each against its own direction


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_iteration_from_host_buffers(cuda, dtype):
    """iteration_host (x and dx copied in, the force copied out inside the
    enqueued and then graph-replayed sequence) gives iteration()'s result
    from device tensors: first call eager, second and third replayed, the
    third with other host contents in the same buffers."""
    sc = small_scenes()[1]
    pipe, dx = _pipe(sc, dtype, cuda)
    ref_pipe, _ = _pipe(sc, dtype, cuda)
    xh = torch.tensor(sc.x, dtype=dtype).pin_memory()
    dxh = dx.cpu().pin_memory()
    bh = torch.empty_like(xh).pin_memory()
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    rng = np.random.default_rng(4)
    for call in range(3):
        if call == 2:  # new contents in the same pinned buffers: the replay must read them
            xh.copy_(torch.tensor(sc.x + rng.normal(scale=0.05 * sc.dhat, size=sc.x.shape), dtype=dtype))
            dxh.mul_(0.5)
        r = pipe.iteration_host(xh, dxh, bh)
        ref_pipe.soup.x_transformed.copy_(xh.to(cuda))
        q = ref_pipe.iteration(dxh.to(cuda))
        assert (r.n_ee, r.n_pt) == (q.n_ee, q.n_pt) and r.n_ee + r.n_pt > 0
        assert r.alpha == q.alpha
        assert r.energy == pytest.approx(q.energy, rel=1e-12 if dtype == torch.float64 else 1e-6)
        b_ref = ref_pipe.b.double().cpu()
        assert (bh.double() - b_ref).abs().max() <= tol * max(b_ref.abs().max().item(), 1e-300)
    assert pipe._graph is not None  # the later calls replayed the captured sequence
