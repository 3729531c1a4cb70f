"""Sparse Cholesky (libipcb200_direct) against scipy on the same BSR (gpu)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

from ipc_warp_b200.bsr import bsr_from_triplets
from ipc_warp_b200.direct import DirectSolver, DirectSolverError

pytestmark = pytest.mark.gpu


def spd_bsr(nb, seed, dtype, cuda, band=6):
    """A symmetric positive definite block matrix with a banded random
    pattern (mass-like diagonal plus Gram-type off-diagonal couplings)."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(nb):
        for j in rng.choice(np.arange(max(0, i - band), i), size=min(i, 3), replace=False) if i else []:
            B = rng.normal(size=(3, 3)) * 0.3
            # couple i and j through a PSD 6x6 term [[B B^T, -B B^T], ...]
            G = B @ B.T
            rows += [i, j, i, j]
            cols += [i, j, j, i]
            vals += [G, G, -G, -G]
    rows += list(range(nb))
    cols += list(range(nb))
    vals += [np.eye(3) * (1.0 + rng.uniform())] * nb
    t = lambda a, dt=None: torch.tensor(np.asarray(a), dtype=dt, device=cuda)
    A = bsr_from_triplets(nb, nb, t(rows, torch.int32), t(cols, torch.int32), t(np.stack(vals), dtype))
    return A


@pytest.mark.parametrize("ordering", ["none", "symrcm", "symamd", "metis"])
@pytest.mark.parametrize("fp64", [False, True])
def test_direct_solve_matches_scipy(cuda, ordering, fp64):
    dt = torch.float64 if fp64 else torch.float32
    A = spd_bsr(2000, 7, dt, cuda)
    rng = np.random.default_rng(1)
    b = rng.normal(size=(2000, 3))
    solver = DirectSolver(ordering)
    x = solver(A, torch.tensor(b, dtype=dt, device=cuda)).double().cpu().numpy()
    S = A.to_scipy().tocsc().astype(np.float64)
    ref = spla.spsolve(S, b.reshape(-1)).reshape(-1, 3)
    tol = 1e-10 if fp64 else 2e-4
    assert np.abs(x - ref).max() <= tol * np.abs(ref).max()
    f, w = solver.sizes()
    assert f > 0


def test_refactor_same_pattern_and_reanalyze(cuda):
    A = spd_bsr(500, 3, torch.float64, cuda)
    s = DirectSolver("metis")
    s.analyze_pattern(A)
    b = torch.randn(500, 3, dtype=torch.float64, device=cuda)
    for scale in (1.0, 2.5):
        B = bsr_from_triplets(500, 500, *(lambda t: (t.rows, t.cols, t.vals * scale))(A.triplets()))
        s.factorize(B)
        x = s.solve(b)
        r = torch.tensor(B.to_scipy() @ x.cpu().numpy().reshape(-1)).reshape(-1, 3) - b.cpu()
        assert float(r.abs().max()) <= 1e-10 * float(b.abs().max())
    # a different pattern needs a new analysis
    C = spd_bsr(700, 4, torch.float64, cuda)
    x = s(C, torch.ones(700, 3, dtype=torch.float64, device=cuda))
    r = C.to_scipy() @ x.cpu().numpy().reshape(-1) - 1.0
    assert np.abs(r).max() <= 1e-9


def test_singular_matrix_is_reported(cuda):
    A = spd_bsr(300, 5, torch.float64, cuda)
    nnz = A.nnz_sync()
    # zero one diagonal block (row 0 has no couplings to the left; keep pattern)
    offs = A.offsets.cpu().numpy()
    cols = A.columns[:nnz].cpu().numpy()
    k = [k for k in range(offs[0], offs[1]) if cols[k] == 0][0]
    A.values[k] = 0.0
    s = DirectSolver("none")
    s.analyze_pattern(A)
    with pytest.raises(DirectSolverError) as e:
        s.factorize(A)
    assert e.value.code == 3
