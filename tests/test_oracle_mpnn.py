"""The learned-preconditioner oracle is self-consistent: the row
normalisation makes every diagonal block of G A^ G^T the identity, its FSAI
loss equals the Kaporin loss of the normalised factor, the backward pass is
the derivative of that loss (finite differences, rounding off) and the
preconditioner it defines is SPD."""
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


def _diag_blocks_of_GAGt(g, Ah, G):
    """(G A^ G^T)_ii for every row."""
    T = om.products(g, Ah, G)
    out = []
    for i, row in enumerate(om._lower_rows(g)):
        out.append(sum(T[s] @ G[s].T for (_, s) in row))
    return np.array(out)


def test_zero_head_gives_first_order_directions_and_normalised_rows():
    g, Ah, s, x, y, _ = _system()
    p = om.init_params(0)
    H = om.forward(g, x, y, p, Ah=Ah)
    isd = g.cols[g.lower] == g.rows[g.lower]
    assert np.allclose(H[isd], np.eye(3))
    assert np.allclose(H[~isd], -Ah.astype(np.float32)[g.lower][~isd])
    G, loss, _ = om.normalize(g, Ah, H)
    assert np.allclose(_diag_blocks_of_GAGt(g, Ah, G), np.eye(3), atol=1e-10)
    assert abs(om.kaporin(g, Ah, G) - loss) < 1e-10
    # Jacobi (G^ = I) has Kaporin loss 0; the normalised first-order factor is below it
    J = np.where(isd[:, None, None], np.eye(3), 0.0)
    assert abs(om.kaporin(g, Ah, J)) < 1e-12 and loss < 0


def test_fsai_loss_gradient_by_finite_differences():
    g, Ah, s, x, y, _ = _system(seed=1)
    rng = np.random.default_rng(2)
    isd = g.cols[g.lower] == g.rows[g.lower]
    H = np.where(isd[:, None, None], np.eye(3), -Ah[g.lower] + 0.05 * rng.normal(size=(len(g.lower), 3, 3)))
    _, loss, dH = om.normalize(g, Ah, H)
    D = rng.normal(size=H.shape) * (~isd)[:, None, None]
    eps = 1e-6
    _, lp, _ = om.normalize(g, Ah, H + eps * D)
    _, lm, _ = om.normalize(g, Ah, H - eps * D)
    fd = (lp - lm) / (2 * eps)
    assert abs(fd - (dH * D).sum()) <= 1e-6 * max(1.0, abs(fd))


def test_parameter_gradients_by_finite_differences(no_rounding):
    g, Ah, s, x, y, _ = _system(nb=16, seed=3)
    p = om.init_params(4, zero_head=False)
    H, cache = om.forward(g, x, y, p, keep=True, Ah=Ah)
    _, loss, dH = om.normalize(g, Ah, H)
    grads = om.backward(g, x, y, p, dH, cache)
    rng = np.random.default_rng(5)
    for name in ["W_hin", "W_ein", "W1_0", "b1_0", "W2_1", "W1_3", "b2_3", "W_off", "b_off"]:
        D = rng.normal(size=p[name].shape)
        eps = 1e-6
        q = dict(p)
        q[name] = p[name] + eps * D
        _, lp, _ = om.normalize(g, Ah, om.forward(g, x, y, q, Ah=Ah))
        q[name] = p[name] - eps * D
        _, lm, _ = om.normalize(g, Ah, om.forward(g, x, y, q, Ah=Ah))
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
