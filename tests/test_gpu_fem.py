"""Tet FEM term (fem/fem.py tet_kernel_sparse, compute_Psi) against the
oracle (gpu)."""
import ctypes

import numpy as np
import pytest
import torch

from ipc_warp_b200 import _native as N
from ipc_warp_b200.scenes import two_cubes
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _deformed(n, seed, noise=0.03):
    """Affine stretch/shear plus per-vertex noise (a fraction of the cell
    size); every tet keeps a positive orientation."""
    sc = two_cubes(n=n, gap=0.2, angle_deg=10.0, jitter=0.0, seed=seed)
    rng = np.random.default_rng(seed)
    A = np.array([[1.2, 0.1, 0.0], [0.0, 0.85, 0.05], [0.02, 0.0, 1.0]])
    x = sc.xcs @ A.T + rng.normal(scale=noise / n, size=sc.xcs.shape)
    X = x[sc.tets]
    Dm0 = sc.xcs[sc.tets]
    d = np.linalg.det(np.stack([X[:, i] - X[:, 3] for i in range(3)], axis=2))
    d0 = np.linalg.det(np.stack([Dm0[:, i] - Dm0[:, 3] for i in range(3)], axis=2))
    assert np.all(d * d0 > 0)
    return sc, x


@pytest.mark.parametrize("material", [0, 1, 2])
@pytest.mark.parametrize("fp64", [False, True])
def test_tet_hessian_force_energy(cuda, material, fp64):
    sc, x = _deformed(4, material + 3 * fp64)
    mu, lam = 3.5e4, 9.0e4
    dt = torch.float64 if fp64 else torch.float32
    tx = torch.tensor(x, dtype=dt, device=cuda)
    txcs = torch.tensor(sc.xcs, dtype=dt, device=cuda)
    tets = torch.tensor(sc.tets, dtype=torch.int32, device=cuda)
    n = tets.shape[0]
    Bm = torch.zeros((n, 3, 3), dtype=dt, device=cuda)
    W = torch.zeros(n, dtype=dt, device=cuda)
    N.call("ipcb_tet_rest", int(fp64), N.ptr(txcs), N.ptr(tets), n, N.ptr(Bm), N.ptr(W), N.stream_handle())
    rows = torch.full((16 * n,), -1, dtype=torch.int32, device=cuda)
    cols = torch.full((16 * n,), -1, dtype=torch.int32, device=cuda)
    vals = torch.zeros((16 * n, 3, 3), dtype=dt, device=cuda)
    b = torch.zeros_like(tx)
    N.call("ipcb_tet_hessian", material, int(fp64), N.ptr(tx), N.ptr(tets), n, N.ptr(Bm), N.ptr(W), mu, lam,
           N.ptr(rows), N.ptr(cols), N.ptr(vals), N.ptr(b), N.stream_handle())
    e = torch.zeros(1, dtype=torch.float64, device=cuda)
    N.call("ipcb_tet_energy", material, int(fp64), N.ptr(tx), N.ptr(tets), n, N.ptr(Bm), N.ptr(W), mu, lam,
           N.ptr(e), N.stream_handle())
    torch.cuda.synchronize()
    xin = tx.double().cpu().numpy()
    force, blocks, energy = po.tet(material, xin, txcs.double().cpu().numpy(), sc.tets, mu, lam)
    T = sc.tets.astype(np.int32)
    assert np.array_equal(rows.cpu().numpy().reshape(n, 4, 4), np.repeat(T[:, :, None], 4, axis=2))
    assert np.array_equal(cols.cpu().numpy().reshape(n, 4, 4), np.repeat(T[:, None, :], 4, axis=1))
    tol = 1e-10 if fp64 else 2e-5
    K = vals.double().cpu().numpy().reshape(n, 16, 3, 3)
    scale = np.abs(blocks).max()
    assert np.abs(K - blocks).max() <= tol * scale
    f = b.double().cpu().numpy()
    assert np.abs(f - force).max() <= tol * np.abs(force).max()
    assert abs(float(e.item()) - energy) <= tol * max(abs(energy), 1.0) * (1 if fp64 else 10)


def test_tet_rest_volumes(cuda):
    sc = two_cubes(n=3, gap=0.2, angle_deg=0.0, jitter=0.0, seed=0)
    txcs = torch.tensor(sc.xcs, dtype=torch.float64, device=cuda)
    tets = torch.tensor(sc.tets, dtype=torch.int32, device=cuda)
    n = tets.shape[0]
    Bm = torch.zeros((n, 3, 3), dtype=torch.float64, device=cuda)
    W = torch.zeros(n, dtype=torch.float64, device=cuda)
    N.call("ipcb_tet_rest", 1, N.ptr(txcs), N.ptr(tets), n, N.ptr(Bm), N.ptr(W), N.stream_handle())
    X = sc.xcs[sc.tets]
    Dm = np.stack([X[:, 0] - X[:, 3], X[:, 1] - X[:, 3], X[:, 2] - X[:, 3]], axis=2)
    assert np.allclose(W.cpu().numpy(), np.abs(np.linalg.det(Dm)) / 6.0, rtol=1e-12)
    assert np.allclose(Bm.cpu().numpy(), np.linalg.inv(Dm), rtol=1e-10, atol=1e-10)
    # two unit-ish cubes: total volume matches the bounding boxes
    body = sc.body
    for bi in np.unique(body):
        idx = np.nonzero(np.isin(sc.tets, np.nonzero(body == bi)[0]).all(axis=1))[0]
        assert W.cpu().numpy()[idx].sum() > 0


@pytest.mark.parametrize("material,code", [("snh", 0), ("neo_hookean", 1), ("stvk", 2)])
@pytest.mark.parametrize("fp64", [False, True])
def test_tet_kernels_match_reference_fixture(cuda, material, code, fp64):
    """The reference's own compute_Dm, tet_kernel_sparse and compute_Psi
    (fem/fem.py:22-35,139-203, time_integrator_base.py:125-137), run at
    fixture time on each material file (tests/golden/fem_tets.npz): the GPU
    kernels on the same inputs, against the reference build of the same
    precision (1e-10 double; 2e-5 float)."""
    import os

    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fem_tets.npz"))
    dt = torch.float64 if fp64 else torch.float32
    key = f"{material}_{64 if fp64 else 32}"
    tx = torch.tensor(d["x"], dtype=dt, device=cuda)
    txcs = torch.tensor(d["xcs"], dtype=dt, device=cuda)
    tets = torch.tensor(d["tets"], dtype=torch.int32, device=cuda)
    n = tets.shape[0]
    mu, lam = float(d["mu"]), float(d["lam"])
    Bm = torch.zeros((n, 3, 3), dtype=dt, device=cuda)
    W = torch.zeros(n, dtype=dt, device=cuda)
    N.call("ipcb_tet_rest", int(fp64), N.ptr(txcs), N.ptr(tets), n, N.ptr(Bm), N.ptr(W), N.stream_handle())
    rows = torch.full((16 * n,), -1, dtype=torch.int32, device=cuda)
    cols = torch.full((16 * n,), -1, dtype=torch.int32, device=cuda)
    vals = torch.zeros((16 * n, 3, 3), dtype=dt, device=cuda)
    b = torch.zeros_like(tx)
    N.call("ipcb_tet_hessian", code, int(fp64), N.ptr(tx), N.ptr(tets), n, N.ptr(Bm), N.ptr(W), mu, lam,
           N.ptr(rows), N.ptr(cols), N.ptr(vals), N.ptr(b), N.stream_handle())
    e = torch.zeros(1, dtype=torch.float64, device=cuda)
    N.call("ipcb_tet_energy", code, int(fp64), N.ptr(tx), N.ptr(tets), n, N.ptr(Bm), N.ptr(W), mu, lam,
           N.ptr(e), N.stream_handle())
    torch.cuda.synchronize()
    tol = 1e-10 if fp64 else 2e-5
    assert np.array_equal(rows.cpu().numpy(), d[key + "_rows"])
    assert np.array_equal(cols.cpu().numpy(), d[key + "_cols"])
    ref = d[key + "_vals"].astype(np.float64)
    assert np.abs(vals.double().cpu().numpy() - ref).max() <= tol * np.abs(ref).max()
    fr = d[key + "_force"].astype(np.float64)
    assert np.abs(b.double().cpu().numpy() - fr).max() <= tol * np.abs(fr).max()
    er = float(d[key + "_psi"].astype(np.float64).sum())
    assert abs(float(e.item()) - er) <= tol * abs(er)
