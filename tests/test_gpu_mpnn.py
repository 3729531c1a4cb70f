"""Learned FSAI preconditioner kernels (graph, features, tcgen05 forward and
backward, Kaporin loss, Adam, preconditioner apply) against the CPU oracle
oracle/mpnn.py (gpu)."""
import numpy as np
import pytest
import torch

from ipc_warp_b200 import learned as L
from ipc_warp_b200.bsr import BsrMatrix
from oracle import mpnn as om

pytestmark = pytest.mark.gpu


def _bsr(offsets, cols, vals, dtype, cuda):
    n = len(offsets) - 1
    A = BsrMatrix(n, n, len(cols), dtype, cuda)
    A.offsets.copy_(torch.tensor(offsets, dtype=torch.int32))
    A.columns.copy_(torch.tensor(cols, dtype=torch.int32))
    A.values.copy_(torch.tensor(vals, dtype=dtype))
    A.nnz_dev.fill_(len(cols))
    return A


def _case(nb, seed, cuda, dtype=torch.float32):
    offsets, cols, vals = om.random_spd(nb, seed)
    g = om.graph(offsets, cols)
    A = _bsr(offsets, cols, vals, dtype, cuda)
    sysm = L.System.from_bsr(A)
    return g, vals, A, sysm


def test_param_layout_matches_oracle():
    assert L.PARAM_COUNT == sum(np.asarray(v).size for v in om.init_params(0).values())
    assert [k for k, _ in L.PARAMS] == om.PARAM_ORDER


@pytest.mark.parametrize("nb", [1, 7, 300])
def test_graph_and_features(cuda, nb):
    g, vals, A, sysm = _case(nb, nb, cuda)
    G = sysm.graph
    assert np.array_equal(G.rows.cpu().numpy(), g.rows)
    assert np.array_equal(G.rev.cpu().numpy(), g.rev)
    assert np.array_equal(G.diag.cpu().numpy(), g.diag)
    assert np.array_equal(G.lower.cpu().numpy(), g.lower)
    Ah, s = om.scaled(g, vals.astype(np.float32))
    assert np.allclose(sysm.scale.cpu().numpy(), s, rtol=1e-6)
    assert np.allclose(sysm.ahat.cpu().numpy().reshape(-1, 3, 3), Ah, rtol=1e-5, atol=1e-6)
    x, y = om.features(g, Ah)
    # same values up to one bf16 ulp where a float rounding difference flips
    assert np.allclose(sysm.x.float().cpu().numpy(), x, rtol=8e-3, atol=1e-6)
    assert np.allclose(sysm.y.float().cpu().numpy(), y, rtol=8e-3, atol=1e-6)


def _oracle_inputs(sysm):
    return sysm.x.float().cpu().numpy().astype(np.float64), sysm.y.float().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("nb", [5, 200, 2000])
def test_forward_matches_oracle(cuda, nb):
    g, vals, A, sysm = _case(nb, 11 + nb, cuda)
    p = om.init_params(3, zero_head=False)
    net = L.Net(L.flatten(p), device=cuda)
    H, _ = L.forward(net, sysm)
    x, y = _oracle_inputs(sysm)
    ref = om.forward(g, x, y, p, Ah=sysm.ahat.cpu().numpy())
    got = H.cpu().numpy()[g.lower]
    isd = g.cols[g.lower] == g.rows[g.lower]
    assert np.array_equal(got[isd], np.tile(np.eye(3), (isd.sum(), 1, 1)))
    fo = -sysm.ahat.cpu().numpy().reshape(-1, 3, 3)[g.lower][~isd]
    dev = np.abs(ref[~isd] - fo).max()
    assert dev > 1e-4  # the trunk and head matter
    assert np.abs(got[~isd] - ref[~isd]).max() <= 3e-2 * dev + 1e-6


def test_zero_head_gives_first_order_fsai(cuda):
    g, vals, A, sysm = _case(100, 2, cuda)
    net = L.Net(device=cuda)
    H, _ = L.forward(net, sysm)
    got = H.cpu().numpy()[g.lower]
    Ah = sysm.ahat.cpu().numpy().reshape(-1, 3, 3)[g.lower]
    ref = np.where((g.cols[g.lower] == g.rows[g.lower])[:, None, None], np.eye(3), -Ah)
    assert np.allclose(got, ref, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("nb", [6, 400])
def test_normalize_loss_and_gradient(cuda, nb):
    """Row normalisation, FSAI loss and the head-output gradient against the
    oracle on the same directions H."""
    g, vals, A, sysm = _case(nb, 21 + nb, cuda)
    rng = np.random.default_rng(nb)
    isd = g.cols[g.lower] == g.rows[g.lower]
    Ahl = sysm.ahat.cpu().numpy().reshape(-1, 3, 3)[g.lower].astype(np.float64)
    Hl = np.where(isd[:, None, None], np.eye(3), -Ahl + 0.05 * rng.normal(size=(len(g.lower), 3, 3)))
    Hfull = np.zeros((len(g.cols), 3, 3), np.float32)
    Hfull[g.lower] = Hl
    nz = L.normalize(sysm, torch.tensor(Hfull, device=cuda))
    assert nz.status == 0
    Ah = sysm.ahat.double().cpu().numpy().reshape(-1, 3, 3)
    Gref, lref, dHref = om.normalize(g, Ah, Hfull[g.lower].astype(np.float64))
    assert abs(nz.loss - lref) <= 1e-5 * max(1.0, abs(lref))
    G = nz.G.cpu().numpy()[g.lower]
    assert np.abs(G - Gref).max() <= 1e-5 * np.abs(Gref).max()
    dG = L.loss_grad(sysm, nz).float().cpu().numpy()
    x, _ = _oracle_inputs(sysm)
    rho = om.coupling(x)[g.rows[g.lower]]
    dref = om.head_output_grad(dHref, isd, Ahl, rho)
    assert np.abs(dG[:, 9:]).max() == 0 and np.abs(dG[isd]).max() == 0
    assert np.abs(dG[:, :9] - dref).max() <= 1e-2 * np.abs(dref).max()


def test_backward_matches_oracle(cuda):
    g, vals, A, sysm = _case(600, 5, cuda)
    p = om.init_params(7, zero_head=False)
    net = L.Net(L.flatten(p), device=cuda)
    H, tape = L.forward(net, sysm, training=True)
    nz = L.normalize(sysm, H)
    dG = L.loss_grad(sysm, nz)
    grad = torch.zeros_like(net.params)
    L.backward(net, sysm, tape, dG, grad)
    got = L.unflatten(grad.cpu().numpy())
    x, y = _oracle_inputs(sysm)
    Ho, cache = om.forward(g, x, y, p, keep=True, Ah=sysm.ahat.cpu().numpy())
    Ah = sysm.ahat.double().cpu().numpy().reshape(-1, 3, 3)
    _, _, dH = om.normalize(g, Ah, Ho)
    ref = om.backward(g, x, y, p, dH, cache)
    for k, _ in L.PARAMS:
        a, b = got[k].ravel().astype(np.float64), ref[k].ravel()
        nb = np.linalg.norm(b)
        if nb < 1e-12:
            assert np.linalg.norm(a) < 1e-6, k
            continue
        cos = float(a @ b) / (np.linalg.norm(a) * nb)
        assert cos > 0.995, (k, cos)
        assert np.linalg.norm(a - b) <= 0.1 * nb, (k, np.linalg.norm(a - b) / nb)


def test_fsai_apply_matches_oracle(cuda):
    for dtype in (torch.float32, torch.float64):
        g, vals, A, sysm = _case(500, 9, cuda, dtype)
        rng = np.random.default_rng(1)
        Gl = np.tile(np.eye(3), (len(g.lower), 1, 1)) + 0.2 * rng.normal(size=(len(g.lower), 3, 3))
        Gfull = np.zeros((len(g.cols), 3, 3), np.float32)
        Gfull[g.lower] = Gl
        r = rng.normal(size=(g.n, 3))
        ap = L._Apply(sysm, torch.tensor(Gfull, device=cuda), dtype)
        z = ap(torch.tensor(r, dtype=dtype, device=cuda)).double().cpu().numpy()
        ref = om.apply_preconditioner(g, Gl.astype(np.float32).astype(np.float64),
                                      sysm.scale.double().cpu().numpy(), r)
        assert np.abs(z - ref).max() <= (1e-5 if dtype == torch.float32 else 1e-12) * np.abs(ref).max()


def test_adam_step(cuda):
    n = 1000
    p = torch.randn(n, device=cuda)
    g = torch.randn(n, device=cuda)
    m = torch.zeros(n, device=cuda)
    v = torch.zeros(n, device=cuda)
    p0 = p.clone()
    from ipc_warp_b200 import _native as N

    N.call("ipcb_adam", n, N.ptr(p), N.ptr(g), N.ptr(m), N.ptr(v), 1e-2, 0.9, 0.999, 1e-8, 1, N.stream_handle())
    # the first bias-corrected step is lr * g / (|g| + eps)
    assert torch.allclose(p, p0 - 1e-2 * g / (g.abs() + 1e-8), atol=1e-6)


def test_training_lowers_kaporin_loss(cuda):
    systems = [_case(400, s, cuda)[3] for s in range(4)]
    net = L.Net(device=cuda, seed=1)
    tr = L.Trainer(net, lr=2e-3)
    first = tr.step(systems)
    for _ in range(60):
        last = tr.step(systems)
    # the zero head is first-order FSAI; training moves the loss below it
    assert last < first - 2e-3, (first, last)
