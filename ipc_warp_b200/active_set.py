"""Hashed active set of the augmented-Lagrangian contact solver
(augmented_lagrangian.py:105-198, 506-572) on the kernels of csrc/alset.cu.

``ActiveSet(contact_volume)`` keeps ``hash`` (an :class:`ALHash`: bucket
starts ``cell_start`` and ``ALConstraint`` columns), ``capacity``,
``count()``, ``create_hash(contacts, n, vertex_toi)`` and ``merge(new)`` as
the reference; ``accumulate_vertex_toi`` is the per-vertex minimum time of
impact that ``create_hash`` filters with.  Records come from
``ContactSolverBase.new_intersections`` (``contacts_new`` / ``contacts_pt``).
The solver that linearises and updates the constraints (RodComplexAL) is not
part of this package.
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N
from .contact import Contacts


class ALHash:
    """augmented_lagrangian.py ``Hash`` + ``ALConstraint`` columns."""

    def __init__(self, contact_volume: int, dtype, device):
        cap = max(1, int(contact_volume))
        self.table_size = max(2, 2 * cap)
        self.capacity = cap
        self.dtype, self.device = dtype, device
        i32 = dict(dtype=torch.int32, device=device)
        sc = dict(dtype=dtype, device=device)
        self.cell_start = torch.zeros(self.table_size + 1, **i32)
        self.a1a2b1b2 = torch.zeros((cap, 4), **i32)
        self.e0e1 = torch.zeros((cap, 2), **i32)
        self.l0, self.alpha, self.lam, self.gamma, self.slack, self.mollifier, self.d0 = (
            torch.zeros(cap, **sc) for _ in range(7))
        self.distance_type = torch.zeros(cap, **i32)
        self.grad = torch.zeros((cap, 12), **sc)

    def c_struct(self) -> N.AlSet:
        p = N.ptr
        return N.AlSet(self.table_size, self.capacity, p(self.cell_start), p(self.a1a2b1b2), p(self.e0e1), p(self.l0),
                       p(self.alpha), p(self.lam), p(self.gamma), p(self.slack), p(self.mollifier), p(self.d0),
                       p(self.distance_type), p(self.grad))

    def count(self) -> int:
        return int(self.cell_start[-1].item())


def accumulate_vertex_toi(contacts: Contacts, n: int, vertex_toi: torch.Tensor):
    """augmented_lagrangian.py:105-113: vertex_toi[v] = min over the first n
    records touching v of their alpha (vertex_toi non-negative on entry)."""
    N.call("ipcb_al_vertex_toi", int(vertex_toi.dtype == torch.float64), ctypes.byref(contacts.c_struct()), int(n),
           N.ptr(vertex_toi), N.stream_handle())


class ActiveSet:
    """augmented_lagrangian.py:506-572 (hash part)."""

    def __init__(self, contact_volume: int, dtype=torch.float32, device="cuda"):
        self.dtype, self.device = dtype, torch.device(device)
        self.hash = self.reserve(max(1, contact_volume))

    def reserve(self, contact_volume: int) -> ALHash:
        return ALHash(contact_volume, self.dtype, self.device)

    @property
    def capacity(self) -> int:
        return self.hash.capacity

    def count(self) -> int:
        return self.hash.count()

    def _ws(self, table_size: int) -> torch.Tensor:
        return torch.empty(N.size("ipcb_al_workspace", table_size), dtype=torch.uint8, device=self.device)

    def create_hash(self, contacts: Contacts, n_constraints: int, vertex_toi: torch.Tensor):
        required = max(1, int(n_constraints))
        if required > self.capacity:
            self.hash = self.reserve(1 << (required - 1).bit_length())
        ws = self._ws(self.hash.table_size)
        N.call("ipcb_al_create", int(self.dtype == torch.float64), ctypes.byref(self.hash.c_struct()),
               ctypes.byref(contacts.c_struct()), int(n_constraints), N.ptr(vertex_toi), N.ptr(ws), ws.numel(),
               N.stream_handle())

    def merge(self, new: "ActiveSet"):
        n_old, n_new = self.count(), new.count()
        destination = self.reserve(max(1, n_old + n_new))
        ws = self._ws(destination.table_size)
        N.call("ipcb_al_merge", int(self.dtype == torch.float64), ctypes.byref(new.hash.c_struct()),
               ctypes.byref(self.hash.c_struct()), ctypes.byref(destination.c_struct()), n_new, n_old, N.ptr(ws),
               ws.numel(), N.stream_handle())
        self.hash = destination
