"""Linear BVH over AABB arrays: the stand-in for ``wp.Bvh`` / ``wp.Mesh``
(contact.py:464-483: built once, ``.refit()`` per query, contact.py:672-677).

``Bvh(lower, upper)`` keeps references to the two float32 (n, 3) box tensors
like ``wp.Bvh`` does, builds the hierarchy on construction (Morton codes,
device radix sort, Karras emission, atomic refit) and exposes ``refit()``
(same topology, new boxes) and ``rebuild()`` (new topology).
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N


class Bvh:
    def __init__(self, lower: torch.Tensor, upper: torch.Tensor, capacity: int | None = None):
        assert lower.dtype == torch.float32 and upper.dtype == torch.float32
        assert lower.shape == upper.shape and lower.shape[-1] == 3
        self.lower, self.upper = lower, upper
        self.device = lower.device
        n = lower.shape[0]
        self.capacity = max(int(capacity or n), 1)
        self._mem = torch.empty(N.size("ipcb_lbvh_bytes", self.capacity), dtype=torch.uint8, device=self.device)
        self._ws = torch.empty(N.size("ipcb_lbvh_build_workspace", self.capacity), dtype=torch.uint8,
                               device=self.device)
        self.c = N.Lbvh()
        N.call("ipcb_lbvh_bind", ctypes.byref(self.c), N.ptr(self._mem), self.capacity)
        self.rebuild()

    @property
    def n(self) -> int:
        return self.c.n

    def _view(self, addr: int, count: int, dtype=torch.int32) -> torch.Tensor:
        off = addr - self._mem.data_ptr()
        nbytes = count * torch.tensor([], dtype=dtype).element_size()
        return self._mem[off:off + nbytes].view(dtype)

    @property
    def sorted(self) -> torch.Tensor:
        """Primitive of each leaf slot (Morton order), int32[n]."""
        return self._view(self.c.sorted, self.c.n)

    @property
    def nodes(self) -> torch.Tensor:
        """Internal nodes as float32[n-1, 4, 4]: (L.lo, Lcode) (L.hi) (R.lo, Rcode) (R.hi)."""
        m = max(self.c.n - 1, 1)
        return self._view(self.c.nodes, 16 * m, torch.float32).view(m, 4, 4)

    @property
    def parent(self) -> torch.Tensor:
        return self._view(self.c.parent, 2 * self.capacity)

    def rebuild(self, lower: torch.Tensor | None = None, upper: torch.Tensor | None = None, stream=None):
        if lower is not None:
            self.lower, self.upper = lower, upper
        n = self.lower.shape[0]
        if n > self.capacity:
            raise ValueError(f"Bvh capacity {self.capacity} < {n} boxes")
        N.call("ipcb_lbvh_build", ctypes.byref(self.c), N.ptr(self.lower), N.ptr(self.upper), n,
               N.ptr(self._ws), self._ws.numel(), N.stream_handle(stream))

    def refit(self, lower: torch.Tensor | None = None, upper: torch.Tensor | None = None, stream=None):
        """Recompute node boxes keeping the topology; by default from the
        bound box arrays, or from other (n, 3) boxes of the same primitives."""
        lo = self.lower if lower is None else lower
        hi = self.upper if upper is None else upper
        assert lo.shape[0] == self.c.n and hi.shape[0] == self.c.n
        N.call("ipcb_lbvh_refit", ctypes.byref(self.c), N.ptr(lo), N.ptr(hi), N.stream_handle(stream))


def sort_pairs(keys: torch.Tensor, vals: torch.Tensor, end_bit: int, stream=None) -> None:
    """In-place stable device radix sort of (keys, vals) by the low end_bit bits."""
    n = keys.numel()
    if keys.dtype == torch.int32:
        ws = torch.empty(N.size("ipcb_sort_workspace_u32", n), dtype=torch.uint8, device=keys.device)
        N.call("ipcb_sort_pairs_u32", N.ptr(keys), N.ptr(vals), n, end_bit, N.ptr(ws), ws.numel(),
               N.stream_handle(stream))
    elif keys.dtype == torch.int64:
        ws = torch.empty(N.size("ipcb_sort_workspace_u64", n), dtype=torch.uint8, device=keys.device)
        N.call("ipcb_sort_pairs_u64", N.ptr(keys), N.ptr(vals), n, end_bit, N.ptr(ws), ws.numel(),
               N.stream_handle(stream))
    else:
        raise TypeError(keys.dtype)
