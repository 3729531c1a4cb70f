"""Direct (sparse Cholesky) solve of the block Newton system: the
``DirectSolverDevice`` surface of the reference's ``solve_ldlt``
(time_integrator_base.py:470-500: ``analyze_pattern``, ``factorize``,
``solve``), backed by libipcb200_direct (include/ipcb_direct.h).

It is the fallback when PCG misses its tolerance and the judge of the
iterative solves.
"""
from __future__ import annotations

import ctypes
import os

import torch

from .bsr import BsrMatrix

_HERE = os.path.dirname(os.path.abspath(__file__))
DIRECT_LIB_PATH = os.path.join(_HERE, "lib", "libipcb200_direct.so")
ORDERINGS = {"none": 0, "symrcm": 1, "symamd": 2, "metis": 3}
IPCB_E_SINGULAR = 3

P, c_int, c_size_t = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
SIGNATURES = {
    "ipcb_direct_last_error": (ctypes.c_char_p, []),
    "ipcb_direct_create": (c_int, [ctypes.POINTER(P)]),
    "ipcb_direct_destroy": (c_int, [P]),
    "ipcb_direct_analyze": (c_int, [P, c_int, c_int, P, P, c_int, c_int, P]),
    "ipcb_direct_factor": (c_int, [P, P, P]),
    "ipcb_direct_solve": (c_int, [P, P, P, P]),
    "ipcb_direct_sizes": (c_int, [P, ctypes.POINTER(c_size_t), ctypes.POINTER(c_size_t)]),
}

_lib = None


def _loaded_dir(soname: str) -> str | None:
    try:
        with open("/proc/self/maps") as f:
            for line in f:
                path = line.rstrip().split(" ")[-1]
                if os.path.basename(path) == soname:
                    return os.path.dirname(path)
    except OSError:
        pass
    return None


def _preload_solver_libs():
    """Load cuSOLVER/cuSPARSE from the family of the cuBLAS torch already
    loaded (its wheel copies or the toolkit's), so that one process never
    resolves two builds of the same soname."""
    from ._build import CUDA_LIB, _solver_lib_dirs

    cublas = _loaded_dir("libcublas.so.12")
    wheel = _solver_lib_dirs()
    if wheel == [CUDA_LIB] or (cublas is not None and "site-packages" not in cublas):
        so_dir = sp_dir = CUDA_LIB
    else:
        so_dir, sp_dir = wheel
    for d, name in ((sp_dir, "libcusparse.so.12"), (so_dir, "libcusolver.so.11")):
        path = os.path.join(d, name)
        if _loaded_dir(name) is None and os.path.exists(path):
            ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(DIRECT_LIB_PATH):
            raise RuntimeError(f"{DIRECT_LIB_PATH} is missing: run ipc_warp_b200/_build.py")
        _preload_solver_libs()
        L = ctypes.CDLL(DIRECT_LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


class DirectSolverError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def _call(name, *args):
    L = lib()
    rc = getattr(L, name)(*args)
    if rc != 0:
        raise DirectSolverError(rc, f"{name} failed ({rc}): {L.ipcb_direct_last_error().decode()}")


class DirectSolver:
    """analyze_pattern / factorize / solve on a canonical BsrMatrix."""

    def __init__(self, ordering: str = "metis"):
        self.ordering = ORDERINGS[ordering]
        h = P()
        _call("ipcb_direct_create", ctypes.byref(h))
        self._h = h
        self._pattern = None
        self.dtype = None

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.ipcb_direct_destroy(self._h)
            self._h = None

    @staticmethod
    def _stream():
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def analyze_pattern(self, A: BsrMatrix):
        nnz = A.nnz_sync()
        _call("ipcb_direct_analyze", self._h, A.nrow, nnz, ctypes.c_void_p(A.offsets.data_ptr()),
              ctypes.c_void_p(A.columns.data_ptr()), int(A.dtype == torch.float64), self.ordering, self._stream())
        self._pattern = (A.nrow, nnz)
        self.dtype = A.dtype

    def factorize(self, A: BsrMatrix):
        if self._pattern is None:
            raise DirectSolverError(1, "factorize before analyze_pattern")
        _call("ipcb_direct_factor", self._h, ctypes.c_void_p(A.values.data_ptr()), self._stream())

    def solve(self, b: torch.Tensor, x: torch.Tensor | None = None) -> torch.Tensor:
        b = b.contiguous()
        if b.dtype != self.dtype:
            raise DirectSolverError(1, "right-hand side type differs from the factor")
        x = torch.empty_like(b) if x is None else x
        _call("ipcb_direct_solve", self._h, ctypes.c_void_p(b.data_ptr()), ctypes.c_void_p(x.data_ptr()),
              self._stream())
        return x

    def sizes(self):
        f, w = c_size_t(), c_size_t()
        _call("ipcb_direct_sizes", self._h, ctypes.byref(f), ctypes.byref(w))
        return f.value, w.value

    def __call__(self, A: BsrMatrix, b: torch.Tensor) -> torch.Tensor:
        """The reference's solve_ldlt: analyze, factorize and solve."""
        self.analyze_pattern(A)
        self.factorize(A)
        return self.solve(b)
