"""One scene's contact iteration split over ranks, checked on one GPU: the
ranks' shares (run one after another, no exchange) add up to the unsharded
ContactPipeline iteration -- the union of their records is its record set,
their forces and energies sum to its, and the smallest of their CCD bounds is
its bound (gpu)."""
import numpy as np
import pytest
import torch

from helpers import small_scenes, sort_records
from ipc_warp_b200.pipeline import ContactPipeline
from ipc_warp_b200.sharded import ShardedContactPipeline

pytestmark = pytest.mark.gpu


def _records(s, n_ee, n_pt):
    return (s.contacts_new.records(n_ee).cpu().numpy(), s.contacts_pt.records(n_pt).cpu().numpy())


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("idx", [0, 2])
def test_shares_add_up_to_the_unsharded_iteration(cuda, world, idx):
    sc = small_scenes()[idx]
    rng = np.random.default_rng(idx + 10 * world)
    dx = torch.tensor(rng.normal(scale=0.3 * sc.dhat, size=sc.x.shape), dtype=torch.float64, device=cuda)
    full = ContactPipeline.from_scene(sc, dtype=torch.float64, device=cuda)
    full.states.dx = dx
    r_full = full.iteration_stepwise()
    ee_full, pt_full = _records(full, r_full.n_ee, r_full.n_pt)
    b_full = full.b.cpu().numpy().copy()
    ee, pt, b, energy, alphas = [], [], 0.0, 0.0, []
    for rank in range(world):
        s = ShardedContactPipeline.from_scene(sc, rank, world, dtype=torch.float64, device=cuda, exchange=False)
        r = s.iteration(dx)
        e_r, p_r = _records(s, r.n_ee, r.n_pt)
        ee.append(e_r)
        pt.append(p_r)
        b = b + s.b.cpu().numpy()
        energy += r.energy
        alphas.append(r.alpha)
        assert r.status == 0
    assert np.array_equal(sort_records(np.concatenate(ee)), sort_records(ee_full))
    assert np.array_equal(sort_records(np.concatenate(pt)), sort_records(pt_full))
    assert len(ee_full) + len(pt_full) > 0
    assert np.abs(b - b_full).max() <= 1e-10 * np.abs(b_full).max()
    assert energy == pytest.approx(r_full.energy, rel=1e-10)
    assert min(alphas) == r_full.alpha


def test_one_rank_is_the_unsharded_iteration(cuda):
    sc = small_scenes()[1]
    rng = np.random.default_rng(3)
    dx = torch.tensor(rng.normal(scale=0.3 * sc.dhat, size=sc.x.shape), dtype=torch.float32, device=cuda)
    full = ContactPipeline.from_scene(sc, dtype=torch.float32, device=cuda)
    full.states.dx = dx
    r_full = full.iteration_stepwise()
    s = ShardedContactPipeline.from_scene(sc, 0, 1, dtype=torch.float32, device=cuda)
    r = s.iteration(dx)
    assert (r.n_ee, r.n_pt) == (r_full.n_ee, r_full.n_pt) == (r.n_ee_total, r.n_pt_total)
    assert r.alpha == r_full.alpha
