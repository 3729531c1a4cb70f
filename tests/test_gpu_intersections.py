"""Intersection check (ipcb_edge_triangle_crossings) against the oracle's
brute-force-equivalent enumeration, and the rest states of the benchmark
scenes free of crossings (gpu)."""
import numpy as np
import pytest
import torch

from helpers import small_scenes
from ipc_warp_b200 import scenes
from ipc_warp_b200.pipeline import ContactPipeline
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _pairs_sorted(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    return p[np.lexsort(p.T[::-1])] if len(p) else p


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("sink", [0.0, 0.02, 0.15])
def test_crossings_match_oracle(cuda, dtype, sink):
    sc = scenes.two_cubes(n=6, gap=1e-3, angle_deg=20.0, seed=1)
    x = sc.x.copy()
    x[sc.body == 1, 1] -= sink  # the upper cube sinks into the lower one
    sc.x = x
    pipe = ContactPipeline.from_scene(sc, dtype=dtype, device=cuda)
    n, pairs = pipe.edge_triangle_crossings(capacity=1 << 16)
    xin = pipe.soup.x_transformed.double().cpu().numpy()
    on, opairs = po.edge_triangle_crossings(xin, sc.edges, sc.triangles)
    assert n == on
    assert np.array_equal(_pairs_sorted(pairs.cpu().numpy()), _pairs_sorted(opairs))
    if sink == 0.0:
        assert n == 0
    else:
        assert n > 10


@pytest.mark.parametrize("idx", range(4))
def test_contact_scenes_match_oracle(cuda, idx):
    """The parity scenes: the first three are intersection-free; the fourth
    (rods 0.3 dhat apart with a 0.2 dhat vertex jitter on both sides)
    interpenetrates by construction, and the GPU finds the oracle's pairs."""
    sc = small_scenes()[idx]
    pipe = ContactPipeline.from_scene(sc, dtype=torch.float32, device=cuda)
    n, pairs = pipe.edge_triangle_crossings(capacity=1 << 16)
    on, opairs = po.edge_triangle_crossings(sc.x.astype(np.float32), sc.edges, sc.triangles)
    assert n == on
    assert np.array_equal(_pairs_sorted(pairs.cpu().numpy()), _pairs_sorted(opairs))
    assert (n == 0) == (idx < 3)


def test_screw_and_nut_is_intersection_free(cuda):
    """The loaded screw-and-nut state (0.4 dhat on the loaded flank) has no
    crossing, and the state moved past the TOI of the driven step has."""
    sc = scenes.screw_and_nut()
    pipe = ContactPipeline.from_scene(sc, dtype=torch.float32, device=cuda)
    assert pipe.edge_triangle_crossings()[0] == 0
    dx = torch.tensor(scenes.screw_direction(sc), dtype=torch.float32, device=cuda)
    alpha = pipe.collision_free_step(dx)
    assert 0.0 < alpha < 1.0
    x0 = pipe.soup.x_transformed.clone()
    pipe.soup.x_transformed.copy_(x0 - alpha * dx)
    assert pipe.edge_triangle_crossings()[0] == 0  # the bound keeps the state clear
    pipe.soup.x_transformed.copy_(x0 - 1.0 * dx)
    n, _ = pipe.edge_triangle_crossings()
    assert n > 0  # the full step drives the loaded flank through the bolt's
