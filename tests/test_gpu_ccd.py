"""CCD: cubic roots and per-pair TOI bit-exact with the oracle; scene TOI never
above the oracle's and within 1e-6 of it (gpu)."""
import numpy as np
import pytest
import torch

from helpers import small_scenes
from oracle import pyoracle as po
from test_gpu_dcd import make_solver

pytestmark = pytest.mark.gpu


def constructed_cubics(n, rng, bound=1.0):
    r = np.sort(rng.uniform(-0.2 * bound, 1.2 * bound, size=(n, 3)), axis=1)
    a0 = rng.uniform(0.1, 5.0, size=n) * rng.choice([-1, 1], size=n)
    coef = np.stack([-r[:, 0] * r[:, 1] * r[:, 2], r[:, 0] * r[:, 1] + r[:, 0] * r[:, 2] + r[:, 1] * r[:, 2],
                     -r.sum(1), np.ones(n)], 1) * a0[:, None]
    return coef, r


def test_cubic_roots_bit_exact(cuda):
    from ipc_warp_b200.ccd import cubic_roots

    rng = np.random.default_rng(0)
    coef, r = constructed_cubics(4000, rng)
    rand = rng.normal(size=(4000, 4))
    quad = rng.normal(size=(500, 4))
    quad[:, 3] = 0.0
    allc = np.concatenate([coef, rand, quad])
    nr, roots, st = cubic_roots(allc, 0.0, 1.0)
    onr, oroots, ost = po.cubic_roots(allc, 0.0, 1.0)
    assert st == ost == 0
    assert np.array_equal(nr.cpu().numpy(), onr)
    g = roots.cpu().numpy()
    for i in range(len(allc)):
        assert np.array_equal(g[i, :onr[i]], oroots[i, :onr[i]])
    # the constructed roots in [0,1] are recovered
    for i in range(len(coef)):
        want = r[i][(r[i] >= 0) & (r[i] <= 1)]
        if len(want) == onr[i]:
            assert np.allclose(oroots[i, :onr[i]], want, atol=1e-7)


def test_pair_collision_time_bit_exact(cuda):
    from ipc_warp_b200.ccd import collision_time

    rng = np.random.default_rng(1)
    n = 3000
    p0 = rng.normal(size=(n, 4, 3))
    p1 = p0 + rng.normal(scale=0.7, size=(n, 4, 3))
    for kind in ("ee", "pt"):
        t, st = collision_time(kind, p0, p1)
        ot = po.collision_time(kind, p0, p1)
        assert st == 0
        assert np.array_equal(t.cpu().numpy(), ot)
        assert (ot < 1).sum() > 50


def test_known_toi_point_onto_triangle(cuda):
    from ipc_warp_b200.ccd import pt_collision_time

    p0 = np.array([[[0.2, 0.2, 1.0], [0, 0, 0], [1, 0, 0], [0, 1, 0]]])
    p1 = p0.copy()
    p1[0, 0, 2] = -1.0
    assert abs(pt_collision_time(p0, p1).item() - 0.5) < 1e-9


@pytest.mark.parametrize("idx", [0, 1, 2])
@pytest.mark.parametrize("fp64", [False, True])
def test_scene_toi(cuda, idx, fp64):
    sc = small_scenes()[idx]
    dtype = torch.float64 if fp64 else torch.float32
    s = make_solver(sc, dtype)
    rng = np.random.default_rng(idx)
    # push body 1 toward body 0 and add noise: some pairs collide within the step
    dx = np.zeros_like(sc.x)
    dx[sc.body == 1] += np.array([0.0, 4.0, 0.0]) * sc.dhat  # x1 = x - dx: body 1 moves toward body 0
    dx += rng.normal(scale=0.3 * sc.dhat, size=dx.shape)
    dxt = torch.tensor(dx, dtype=dtype, device=cuda)
    alpha = s.collision_free_step(dxt)
    toi = float(s.ccd_toi.item())
    assert s.status == 0
    x0 = s.soup.x_transformed.cpu().numpy()
    x1 = s.ccd_x1.cpu().numpy()
    assert np.array_equal(x1, (x0 - dxt.cpu().numpy()))
    oto, ost = po.scene_toi(x0, x1, sc.edges, sc.triangles, sc.body, fp64=fp64)
    assert ost == 0
    assert oto < 1.0
    assert toi <= oto
    assert oto - toi <= 1e-6
    assert alpha == pytest.approx(0.9 * toi)


def test_no_motion_gives_one(cuda):
    sc = small_scenes()[0]
    s = make_solver(sc)
    alpha = s.collision_free_step(torch.zeros_like(s.soup.x_transformed))
    assert alpha == 1.0


@pytest.mark.parametrize("fp64", [False, True])
def test_small_candidate_list_gives_the_same_toi(cuda, fp64):
    """Candidates that do not fit the staging list send the query to the
    in-place pass: the bound does not depend on the workspace size."""
    sc = small_scenes()[1]
    dtype = torch.float64 if fp64 else torch.float32
    s = make_solver(sc, dtype)
    rng = np.random.default_rng(5)
    dx = np.zeros_like(sc.x)
    dx[sc.body == 1] += np.array([0.0, 4.0, 0.0]) * sc.dhat
    dx += rng.normal(scale=0.3 * sc.dhat, size=dx.shape)
    dxt = torch.tensor(dx, dtype=dtype, device=cuda)
    full = s.collision_free_step(dxt)
    toi_full = float(s.ccd_toi.item())
    from ipc_warp_b200 import _native as N

    s._toi_ws = torch.empty(N.size("ipcb_toi_workspace", 16), dtype=torch.uint8, device=cuda)  # 16 staged pairs
    small = s.collision_free_step(dxt)
    assert float(s.ccd_toi.item()) == toi_full and small == full
    s._toi_ws = torch.empty(N.size("ipcb_toi_workspace", 0), dtype=torch.uint8, device=cuda)  # nothing staged
    assert s.collision_free_step(dxt) == full


def test_pair_times_match_reference_float64_build(cuda):
    """Per-pair times on the float32 inputs of tests/golden/fp32_build.npz
    (random and near-contact motions) equal the reference's float64 build
    run at fixture time, bit for bit; the reference's float32 build is
    compared in test_golden.py."""
    import os

    from ipc_warp_b200.ccd import collision_time

    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fp32_build.npz"))
    for name, kinds in (("random", ("ee", "pt")), ("near_ee", ("ee",)), ("near_pt", ("pt",))):
        p0, p1 = d[name + "_p0"].astype(np.float64), d[name + "_p1"].astype(np.float64)
        for kind in kinds:
            t, st = collision_time(kind, p0, p1)
            assert st == 0
            assert np.array_equal(t.cpu().numpy(), d[f"{name}_t_{kind}64"]), (name, kind)
