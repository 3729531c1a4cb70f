"""3x3-block sparse matrices: the subset of ``warp.sparse`` the Newton
system uses (``bsr_from_triplets``, ``bsr_axpy``, ``bsr_mv``; reference
dynamic_contacts.py:290-297, time_integrator_base.py:406-426,461) and the
``Triplets`` struct of fem/fem.py:15-19.

Assembly sorts (row, col) keys on the device, sums duplicates in input order
and drops all-zero input blocks (as warp's ``prune_numerical_zeros``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N


@dataclass
class Triplets:
    rows: torch.Tensor  # int32 (n,)
    cols: torch.Tensor  # int32 (n,)
    vals: torch.Tensor  # scalar (n, 3, 3)
    # contact triplets only: per record (16 triplets) a 16-bit mask of the
    # blocks with a non-zero entry, int16 (n // 16,)
    mask: torch.Tensor | None = None

    @staticmethod
    def zeros(n: int, dtype, device) -> "Triplets":
        return Triplets(torch.zeros(n, dtype=torch.int32, device=device),
                        torch.zeros(n, dtype=torch.int32, device=device),
                        torch.zeros((n, 3, 3), dtype=dtype, device=device),
                        torch.zeros(max(n // 16, 1), dtype=torch.int16, device=device))


class BsrMatrix:
    def __init__(self, nrow: int, ncol: int, capacity: int, dtype, device):
        self.nrow, self.ncol = int(nrow), int(ncol)
        self.dtype, self.device = dtype, device
        cap = max(int(capacity), 1)
        self.offsets = torch.zeros(self.nrow + 1, dtype=torch.int32, device=device)
        self.columns = torch.zeros(cap, dtype=torch.int32, device=device)
        self.values = torch.zeros((cap, 3, 3), dtype=dtype, device=device)
        self.nnz_dev = torch.zeros(1, dtype=torch.int32, device=device)
        self._ws = None  # contact_bsr workspace, kept between calls

    @property
    def shape(self):
        return (self.nrow, self.ncol)

    def nnz_sync(self) -> int:
        return int(self.nnz_dev.item())

    def to_scipy(self):
        import scipy.sparse as sp

        nnz = self.nnz_sync()
        return sp.bsr_matrix((self.values[:nnz].cpu().numpy(), self.columns[:nnz].cpu().numpy(),
                              self.offsets.cpu().numpy()), shape=(3 * self.nrow, 3 * self.ncol))

    def triplets(self) -> Triplets:
        nnz = self.nnz_sync()
        counts = (self.offsets[1:] - self.offsets[:-1]).long()
        rows = torch.repeat_interleave(torch.arange(self.nrow, device=self.device, dtype=torch.int32), counts)
        return Triplets(rows, self.columns[:nnz].clone(), self.values[:nnz].clone())


def bsr_from_triplets(nrow: int, ncol: int, rows: torch.Tensor, cols: torch.Tensor, vals: torch.Tensor,
                      count: int | None = None, out: BsrMatrix | None = None) -> BsrMatrix:
    n = int(rows.shape[0] if count is None else count)
    dtype = vals.dtype
    dev = vals.device
    if out is None or out.columns.shape[0] < max(n, 1) or out.nrow != nrow:
        out = BsrMatrix(nrow, ncol, n, dtype, dev)
    ws = torch.empty(N.size("ipcb_bsr_workspace", n, nrow, ncol), dtype=torch.uint8, device=dev)
    N.call("ipcb_bsr_from_triplets", nrow, ncol, n, N.ptr(rows), N.ptr(cols), N.ptr(vals),
           int(dtype == torch.float64), N.ptr(out.offsets), N.ptr(out.columns), N.ptr(out.values),
           N.ptr(out.nnz_dev), N.ptr(ws), ws.numel(), N.stream_handle())
    return out


def contact_bsr(ee, n_ee: int | None, pt, n_pt: int | None, n_verts: int, trip: Triplets,
                out: BsrMatrix | None = None, status: torch.Tensor | None = None,
                read_status: bool = True) -> tuple[BsrMatrix, int | None]:
    """BSR of the contact Hessian from the EE/PT lists and their triplets
    (16 blocks per record, EE first, with block masks).  Returns (matrix, status);
    status has IPCB_STATUS_ROW_OVERFLOW (4) set when a row had too many
    distinct columns for the fast path (the matrix is then incomplete).
    n_ee / n_pt None: the lists' counts are read on the device (sizes follow
    the capacities).  read_status=False: no host read; the status stays in
    ``status`` (device) and None is returned in its place."""
    vals = trip.vals
    dtype, dev = vals.dtype, vals.device
    ne = ee.capacity if n_ee is None else n_ee
    npt = pt.capacity if n_pt is None else n_pt
    cap = max(16 * (ne + npt), 1)
    if out is None or out.columns.shape[0] < cap or out.nrow != n_verts or out.dtype != dtype:
        out = BsrMatrix(n_verts, n_verts, cap, dtype, dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev) if status is None else status.zero_()
    nbytes = N.size("ipcb_contact_bsr_workspace", ne + npt, n_verts)
    ws = getattr(out, "_ws", None)
    if ws is None or ws.numel() < nbytes:
        ws = out._ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    import ctypes

    N.call("ipcb_contact_bsr", ctypes.byref(ee.c_struct()), -1 if n_ee is None else n_ee,
           ctypes.byref(pt.c_struct()), -1 if n_pt is None else n_pt, n_verts,
           N.ptr(vals), N.ptr(trip.mask), int(dtype == torch.float64), N.ptr(out.offsets), N.ptr(out.columns),
           N.ptr(out.values), N.ptr(out.nnz_dev), N.ptr(st), N.ptr(ws), ws.numel(), N.stream_handle())
    return out, (int(st.item()) if read_status else None)


def bsr_axpy(x: BsrMatrix, y: BsrMatrix, alpha: float = 1.0, beta: float = 1.0) -> BsrMatrix:
    """y = alpha * x + beta * y on the union pattern (returns the new y)."""
    tx, ty = x.triplets(), y.triplets()
    rows = torch.cat([tx.rows, ty.rows])
    cols = torch.cat([tx.cols, ty.cols])
    vals = torch.cat([tx.vals * alpha, ty.vals * beta])
    return bsr_from_triplets(y.nrow, y.ncol, rows, cols, vals)


def bsr_mv(A: BsrMatrix, x: torch.Tensor, y: torch.Tensor | None = None, alpha: float = 1.0,
           beta: float = 0.0) -> torch.Tensor:
    if y is None:
        y = torch.zeros((A.nrow, 3), dtype=A.dtype, device=A.device)
        beta = 0.0
    N.call("ipcb_bsr_mv", A.nrow, N.ptr(A.offsets), N.ptr(A.columns), N.ptr(A.values),
           int(A.dtype == torch.float64), N.ptr(x), N.ptr(y), float(alpha), float(beta), N.stream_handle())
    return y


def bsr_to_scalar_csr(A: BsrMatrix):
    """time_integrator_base.py:33-62 layout (scalar CSR of the block matrix),
    host-side for the direct solver reference."""
    return A.to_scipy().tocsr()


def scipy_from_triplets(nrow, ncol, rows, cols, vals):
    """Reference assembly on the host (used by tests)."""
    import scipy.sparse as sp

    rows = np.asarray(rows)
    cols = np.asarray(cols)
    vals = np.asarray(vals, dtype=np.float64).reshape(-1, 3, 3)
    keep = np.any(vals != 0, axis=(1, 2))
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    r = (3 * rows[:, None, None] + np.arange(3)[None, :, None]).repeat(3, axis=2)
    c = (3 * cols[:, None, None] + np.arange(3)[None, None, :]).repeat(3, axis=1)
    return sp.coo_matrix((vals.ravel(), (r.ravel(), c.ravel())), shape=(3 * nrow, 3 * ncol)).tocsr()
