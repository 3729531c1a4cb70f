"""The learned-preconditioner oracle is self-consistent: its backward pass is
the derivative of its Kaporin loss (finite differences, rounding off), the
loss is 0 at the Jacobi factor and the preconditioner it defines is SPD."""
import numpy as np
import pytest

from oracle import mpnn as om


@pytest.fixture
def no_rounding():
    om.ROUND = False
    yield
    om.ROUND = True


def _system(nb=24, seed=0):
    offsets, cols, vals = om.random_spd(nb, seed)
    g = om.graph(offsets, cols)
    Ah, s = om.scaled(g, vals)
    x, y = om.features(g, Ah)
    return g, Ah, s, x, y, vals


def test_jacobi_start_has_zero_loss():
    g, Ah, s, x, y, _ = _system()
    p = om.init_params(0)
    G = om.forward(g, x, y, p)
    assert np.allclose(G[g.cols[g.lower] == g.rows[g.lower]], np.eye(3))
    assert np.allclose(G[g.cols[g.lower] != g.rows[g.lower]], 0.0)
    loss, _, _ = om.loss_and_grad_G(g, Ah, G)
    assert abs(loss) < 1e-12


def test_loss_gradient_in_G_by_finite_differences():
    g, Ah, s, x, y, _ = _system(seed=1)
    rng = np.random.default_rng(2)
    G = np.tile(np.eye(3), (len(g.lower), 1, 1)) + 0.1 * rng.normal(size=(len(g.lower), 3, 3))
    _, dG, _ = om.loss_and_grad_G(g, Ah, G)
    D = rng.normal(size=G.shape)
    eps = 1e-6
    lp, _, _ = om.loss_and_grad_G(g, Ah, G + eps * D)
    lm, _, _ = om.loss_and_grad_G(g, Ah, G - eps * D)
    assert abs((lp - lm) / (2 * eps) - (dG * D).sum()) <= 1e-6 * max(1.0, abs((dG * D).sum()))


def test_parameter_gradients_by_finite_differences(no_rounding):
    g, Ah, s, x, y, _ = _system(nb=16, seed=3)
    p = om.init_params(4, zero_head=False)
    G, cache = om.forward(g, x, y, p, keep=True)
    loss, dG, _ = om.loss_and_grad_G(g, Ah, G)
    grads = om.backward(g, x, y, p, dG, cache)
    rng = np.random.default_rng(5)
    for name in ["W_hin", "W_ein", "W1_0", "b1_0", "W2_1", "W1_3", "b2_3", "W_off", "W_dg", "b_dg"]:
        D = rng.normal(size=p[name].shape)
        eps = 1e-6
        q = dict(p)
        q[name] = p[name] + eps * D
        lp, _, _ = om.loss_and_grad_G(g, Ah, om.forward(g, x, y, q))
        q[name] = p[name] - eps * D
        lm, _, _ = om.loss_and_grad_G(g, Ah, om.forward(g, x, y, q))
        fd = (lp - lm) / (2 * eps)
        an = float((grads[name] * D).sum())
        assert abs(fd - an) <= 1e-5 * max(1e-3, abs(fd)), (name, fd, an)


def test_preconditioner_is_spd_and_matches_dense():
    g, Ah, s, x, y, vals = _system(seed=6)
    rng = np.random.default_rng(7)
    G = np.tile(np.eye(3), (len(g.lower), 1, 1)) + 0.2 * rng.normal(size=(len(g.lower), 3, 3))
    n = g.n
    Gd = np.zeros((3 * n, 3 * n))
    for k, e in enumerate(g.lower):
        i, j = g.rows[e], g.cols[e]
        Gd[3 * i:3 * i + 3, 3 * j:3 * j + 3] = G[k]
    S = np.diag(s.reshape(-1))
    Minv = S @ Gd.T @ Gd @ S
    r = rng.normal(size=(n, 3))
    z = om.apply_preconditioner(g, G, s, r)
    assert np.allclose(z.reshape(-1), Minv @ r.reshape(-1))
    assert np.all(np.linalg.eigvalsh(Minv) > 0)
