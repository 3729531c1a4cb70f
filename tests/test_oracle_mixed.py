"""The mixed FEM + affine-body oracle is self-consistent: its gradient is
the derivative of its energy (central differences, float64), its contact
gradient and matrix are J^T of the vertex-space ones, its matrix is
symmetric positive definite, the Jacobian maps q to the vertex positions,
and fixed bodies get no unknown coupling."""
import numpy as np

from ipc_warp_b200 import scenes
from oracle import mixed as om
from oracle import newton as on


def _state(seed=0):
    sc = scenes.mixed_touching()
    p, m, q = om.from_scene(sc)
    rng = np.random.default_rng(seed)
    d = 2e-5 * rng.normal(size=q.shape)
    for b in np.flatnonzero(m.fixed):
        d[m.n_fem + 4 * b:m.n_fem + 4 * b + 4] = 0
    q = q + d
    xt_f = q[:m.n_fem] + 1e-4 * rng.normal(size=(m.n_fem, 3))
    qt_a = q[m.n_fem:] + 1e-4 * rng.normal(size=(4 * m.nb, 3))
    return p, m, q, xt_f, qt_a


def test_jacobian_maps_unknowns_to_vertices():
    sc = scenes.mixed_touching()
    p, m, q = om.from_scene(sc)
    x = om.vertex_positions(m, q)
    world = np.concatenate([sc.fem.x] + [v for v, _ in sc.bodies])
    assert np.abs(x - world).max() < 1e-12


def test_gradient_is_energy_derivative():
    """Elastic, inertia, orthogonality and pin terms by central differences.
    The barrier is switched off (kappa = 0): like the reference it reads the
    float32 closest-point distance, so its energy is quantised at float32
    resolution of the positions (its derivatives are checked per feature
    in test_oracle.py)."""
    p, m, q, xt_f, qt_a = _state()
    p.kappa = 0.0
    g, A, ne, npt = om.system(p, m, q, xt_f, qt_a)
    assert ne + npt > 0
    rng = np.random.default_rng(3)
    for k in range(3):
        d = rng.normal(size=q.shape)
        for b in np.flatnonzero(m.fixed):
            d[m.n_fem + 4 * b:m.n_fem + 4 * b + 4] = 0
        d /= np.abs(d).max()
        eps = 1e-7
        fd = (om.energy(p, m, q + eps * d, xt_f, qt_a) - om.energy(p, m, q - eps * d, xt_f, qt_a)) / (2 * eps)
        an = float((g * d).sum())
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1.0), (k, fd, an)


def test_contact_terms_are_pulled_back_vertex_terms():
    p, m, q, xt_f, qt_a = _state(2)
    g1, A1, ne, npt = om.system(p, m, q, xt_f, qt_a)
    kappa = p.kappa
    p.kappa = 0.0
    g0, A0, _, _ = om.system(p, m, q, xt_f, qt_a)
    p.kappa = kappa
    assert ne + npt > 0
    # vertex-space contact force and Hessian, straight from the narrow phase
    x = om.vertex_positions(m, q)
    ee, pt, l0 = on._contacts(p, x)
    V = len(m.rest)
    f = np.zeros((V, 3))
    H = np.zeros((3 * V, 3 * V))
    for idx, F, Hr, _ in on._narrow(p, x, ee, pt, l0):
        for r in range(len(idx)):
            dofs = (3 * idx[r][:, None] + np.arange(3)).reshape(-1)
            H[np.ix_(dofs, dofs)] += Hr[r]
            for k in range(4):
                f[idx[r, k]] += F[r, 3 * k:3 * k + 3]
    J = om.jacobian(m).toarray()
    h2 = p.h * p.h
    assert np.abs((g1 - g0).reshape(-1) + h2 * J.T @ f.reshape(-1)).max() <= 1e-12 * max(np.abs(g1).max(), 1.0)
    assert np.abs((A1 - A0).toarray() - h2 * J.T @ H @ J).max() <= 1e-12 * np.abs(A1).max()


def test_matrix_symmetric_positive_definite_and_fixed_bodies_decoupled():
    p, m, q, xt_f, qt_a = _state(1)
    g, A, _, _ = om.system(p, m, q, xt_f, qt_a)
    D = A.toarray()
    assert np.abs(D - D.T).max() <= 1e-12 * np.abs(D).max()
    f = m.n_fem + 4 * int(np.flatnonzero(m.fixed)[0])
    blk = D[3 * f:3 * f + 12]
    assert np.allclose(blk[:, 3 * f:3 * f + 12], np.eye(12))
    assert np.abs(np.delete(blk, np.s_[3 * f:3 * f + 12], axis=1)).max() == 0
    free = np.ones(len(D), bool)
    free[3 * f:3 * f + 12] = False
    assert np.linalg.eigvalsh(D[np.ix_(free, free)]).min() > 0
