"""The affine-body oracle is self-consistent: its gradient and Hessian are
the derivatives of its energy (finite differences), the vertex->affine
reductions equal J^T f and J^T H J with the explicit affine Jacobian, the
mass properties of closed surfaces match their analytic values, and the
host-side mass code of the package agrees with the oracle."""
import numpy as np

from ipc_warp_b200 import abd as pabd
from ipc_warp_b200 import scenes
from oracle import abd as oa


def _bodies(nb=3, seed=0):
    rng = np.random.default_rng(seed)
    q = np.zeros((nb, 4, 3))
    q[:, 0] = rng.normal(size=(nb, 3))
    q[:, 1:] = np.eye(3) + 0.1 * rng.normal(size=(nb, 3, 3))
    qt = q + 0.01 * rng.normal(size=q.shape)
    M = np.zeros((nb, 4, 4))
    for b in range(nb):
        C = rng.normal(size=(10, 4))
        C[:, 0] = 1.0
        M[b] = C.T @ C
    vol = rng.uniform(0.5, 2.0, nb)
    stiff = rng.uniform(1e2, 1e3, nb)
    return q, qt, M, vol, stiff


def _energy(q, qt, M, vol, stiff, fixed, h2):
    i, o = oa.body_energy(q, qt, M, vol, stiff, fixed, h2)
    return i + o


def test_body_gradient_and_hessian_by_finite_differences():
    q, qt, M, vol, stiff = _bodies()
    fixed = np.array([0, 0, 1])
    h2 = 1e-4
    blocks, grad = oa.body_system(q, qt, M, vol, stiff, fixed, h2)
    rng = np.random.default_rng(1)
    D = rng.normal(size=q.shape)
    D[fixed == 1] = 0.0
    eps = 1e-6
    fd = (_energy(q + eps * D, qt, M, vol, stiff, fixed, h2) - _energy(q - eps * D, qt, M, vol, stiff, fixed, h2)) / (
        2 * eps)
    assert abs(fd - (grad * D).sum()) <= 1e-6 * max(1.0, abs(fd))
    # Hessian: directional derivative of the gradient
    _, gp = oa.body_system(q + eps * D, qt, M, vol, stiff, fixed, h2)
    _, gm = oa.body_system(q - eps * D, qt, M, vol, stiff, fixed, h2)
    fdg = (gp - gm) / (2 * eps)
    Hd = np.einsum("bijxy,bjy->bix", blocks, D)
    free = fixed == 0
    assert np.abs(fdg[free] - Hd[free]).max() <= 1e-6 * np.abs(Hd).max()
    # fixed body: identity diagonal blocks, zero gradient
    assert np.allclose(blocks[2], np.einsum("ij,xy->ijxy", np.eye(4), np.eye(3)))
    assert np.all(grad[2] == 0)


def test_reductions_equal_jacobian_products():
    rng = np.random.default_rng(3)
    nb, V = 3, 20
    body = np.sort(rng.integers(0, nb, V))
    rest = rng.normal(size=(V, 3))
    fixed = np.array([0, 1, 0])
    J = oa.jacobian(rest, body, nb, fixed)
    f = rng.normal(size=(V, 3))
    assert np.allclose(oa.reduce_force(f, rest, body, fixed, nb).reshape(-1), J.T @ f.reshape(-1))
    n = 30
    rows = rng.integers(0, V, n)
    cols = rng.integers(0, V, n)
    vals = rng.normal(size=(n, 3, 3))
    Hv = oa.dense(rows, cols, vals, V)
    R, C, Vb = oa.reduce_hessian(rows, cols, vals, rest, body, fixed, 0.5)
    assert np.allclose(oa.dense(R, C, Vb, 4 * nb), 0.5 * J.T @ Hv @ J)


def test_affine_map_is_the_jacobian():
    rng = np.random.default_rng(4)
    nb, V = 2, 9
    body = rng.integers(0, nb, V)
    rest = rng.normal(size=(V, 3))
    q = rng.normal(size=(nb, 4, 3))
    J = oa.jacobian(rest, body, nb)
    assert np.allclose(oa.affine_map(q, rest, body).reshape(-1), J @ q.reshape(-1))


def test_mass_properties_of_closed_surfaces():
    v, f = scenes.box_surface((3, 2, 4), (1.0, 2.0, 3.0))
    body = np.zeros(len(v), np.int32)
    c, vol, w = oa.mass_properties(v, f, body)
    assert abs(vol[0] - 6.0) < 1e-12 and np.allclose(c[0], [0.5, 1.0, 1.5])
    assert abs(w.sum() - 2 * (2 + 3 + 6)) < 1e-9  # total surface area
    v, f = scenes.icosphere(3, 0.5)
    body = np.zeros(len(v), np.int32)
    c, vol, w = oa.mass_properties(v, f, body)
    assert np.abs(c).max() < 1e-12
    M = oa.mass_moments(v - c[0], body, w, vol, 1000.0)
    m = 1000.0 * vol[0]
    assert abs(M[0, 0, 0] - m) < 1e-9 * m
    # area-weighted second moments of a sphere: m r^2 / 3 on the diagonal
    assert np.allclose(np.diag(M[0, 1:, 1:]), m * 0.25 / 3, rtol=2e-2)


def test_package_mass_code_matches_oracle():
    cfg = scenes.abd_balls(n_side=2, subdiv=1)
    xs, fs, bs = [], [], []
    off = 0
    for b, ((v, f), T) in enumerate(zip(cfg["meshes"], cfg["transforms"])):
        xs.append(v @ T[:3, :3].T + T[:3, 3])
        fs.append(f + off)
        bs.append(np.full(len(v), b))
        off += len(v)
    x, f, body = np.concatenate(xs), np.concatenate(fs), np.concatenate(bs)
    c1, v1, w1 = pabd.mass_properties(x, f, body)
    c2, v2, w2 = oa.mass_properties(x, f, body)
    assert np.allclose(c1, c2) and np.allclose(v1, v2) and np.allclose(w1, w2)
    M1 = pabd.mass_moments(x - c1[body], body, w1, v1, 1000.0)
    M2 = oa.mass_moments(x - c2[body], body, w2, v2, 1000.0)
    assert np.allclose(M1, M2)
