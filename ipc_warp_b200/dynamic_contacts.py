"""Barrier energy, force and PSD-filtered Hessian per contact record: the
launch surface of dynamic_contacts.py (reference dynamic_contacts.py:152-398).

``contact_hessian_ee(states, soup, contacts, triplets, b, kappa)`` and
``contact_hessian_pt(states, soup, contacts, triplets, b, offset, kappa)``
keep the reference argument order (they are the kernels ABD re-launches,
affine_body_dynamics.py:468-483); ``n`` defaults to the count the last
``detect_collision`` found.  ``b`` accumulates the force (-gradient),
``triplets`` receives 16 3x3 blocks per record at ``(offset + i) * 16 + ii * 4
+ jj``.  :class:`ContactBarrierMixin` adds the RodComplexBC contact parts
(``compute_contact_hessian`` = the contact block of compute_A,
``compute_collision_energy``, ``line_search_upper_bound``).
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N
from .bsr import BsrMatrix, Triplets, bsr_from_triplets, contact_bsr
from .contact import ContactSolverBase, Contacts, Soup


def _count(contacts: Contacts, n):
    return int(contacts.cnt.item()) if n is None else int(n)


def hessian_workspace(contacts: Contacts, ws: torch.Tensor | None) -> torch.Tensor:
    """Device workspace of the class-sorted narrow phase for ``contacts``
    (reused when ``ws`` is large enough)."""
    need = N.size("ipcb_contact_hessian_workspace", contacts.capacity)
    if ws is None or ws.numel() < need:
        ws = torch.empty(need, dtype=torch.uint8, device=contacts.device)
    return ws


def _hessian(kind, soup, contacts, triplets, b, kappa, n, offset, offset_count, ws):
    args = (kind, ctypes.byref(soup.c_struct()), ctypes.byref(contacts.c_struct()), n, int(offset))
    tail = (float(kappa), N.ptr(triplets.rows), N.ptr(triplets.cols), N.ptr(triplets.vals), N.ptr(b),
            N.ptr(triplets.mask))
    if ws is None:
        N.call("ipcb_contact_hessian_after", *args, offset_count, *tail, N.stream_handle())
    else:
        N.call("ipcb_contact_hessian_sorted", *args, offset_count, *tail, N.ptr(ws), ws.numel(), N.stream_handle())


def contact_hessian_ee(states, soup: Soup, contacts: Contacts, triplets: Triplets, b: torch.Tensor, kappa: float,
                       n: int | None = None, ws: torch.Tensor | None = None):
    """dynamic_contacts.py:151-207 (EE with mollifier).  With ``ws``
    (hessian_workspace) the records run in cost-class order."""
    n = n if n is not None and n < 0 else min(_count(contacts, n), contacts.capacity)
    _hessian(0, soup, contacts, triplets, b, kappa, n, 0, None, ws)


def contact_hessian_pt(states, soup: Soup, contacts: Contacts, triplets: Triplets, b: torch.Tensor, offset: int,
                       kappa: float, n: int | None = None, ws: torch.Tensor | None = None):
    """dynamic_contacts.py:209-246 (PT, records at offset)."""
    n = min(_count(contacts, n), contacts.capacity)
    _hessian(1, soup, contacts, triplets, b, kappa, n, offset, None, ws)


def contact_hessian_pt_after(states, soup: Soup, contacts: Contacts, triplets: Triplets, b: torch.Tensor,
                             ee: Contacts, kappa: float, ws: torch.Tensor | None = None):
    """contact_hessian_pt with both counts read on the device: the PT records
    go right after the EE list's min(count, capacity) records, as
    contact_hessian_pt(..., offset=n_ee) puts them, without a host read."""
    _hessian(1, soup, contacts, triplets, b, kappa, -1, ee.capacity, N.ptr(ee.cnt), ws)


def contact_energy_ee(states, soup: Soup, contacts: Contacts, e: torch.Tensor, kappa: float, n: int | None = None):
    """dynamic_contacts.py:374-388; e is a float64 (1,) accumulator."""
    n = min(_count(contacts, n), contacts.capacity)
    N.call("ipcb_contact_energy", 0, ctypes.byref(soup.c_struct()), ctypes.byref(contacts.c_struct()), n,
           float(kappa), N.ptr(e), N.stream_handle())


def contact_energy_pt(states, soup: Soup, contacts: Contacts, e: torch.Tensor, kappa: float, n: int | None = None):
    """dynamic_contacts.py:390-398."""
    n = min(_count(contacts, n), contacts.capacity)
    N.call("ipcb_contact_energy", 1, ctypes.byref(soup.c_struct()), ctypes.byref(contacts.c_struct()), n,
           float(kappa), N.ptr(e), N.stream_handle())


class ContactBarrierMixin(ContactSolverBase):
    """Contact parts of RodComplexBC (dynamic_contacts.py:249-308).

    Expects ``self.soup``, ``self.b`` (force accumulator, (V, 3) scalar),
    ``self.h`` (time step), ``self.contact_stiffness`` (kappa) and optionally
    ``self.states`` (anything; positions come from soup.x_transformed)."""

    def line_search_upper_bound(self):
        return self.collision_free_step(self.states.dx)

    def compute_contact_hessian(self, detect: bool = True, build_bsr: bool = True) -> BsrMatrix | None:
        """The contact block of compute_A (dynamic_contacts.py:275-297):
        detect, then 16 triplets per record and b += force; returns the
        canonical BSR of the contact Hessian (not yet scaled by h^2), or None
        with ``build_bsr=False`` (the caller assembles ``collision_triplets``
        together with its own terms)."""
        if detect:
            with self.profile_timer("detect collision"):
                self.detect_collision()
        with self.profile_timer("compute contact hessian"):
            n_ee, n_pt = self.n_contacts, self.n_contacts_pt
            nnz = (n_ee + n_pt) * 16
            if getattr(self, "collision_triplets", None) is None or self.collision_triplets.rows.shape[0] < nnz:
                self.collision_triplets = Triplets.zeros(max(nnz, 16), self.soup.xcs.dtype, self.device)
            t = self.collision_triplets
            states = getattr(self, "states", None)
            kappa = float(self.contact_stiffness)
            if n_ee:
                self._ws_ee = hessian_workspace(self.contacts_new, getattr(self, "_ws_ee", None))
                contact_hessian_ee(states, self.soup, self.contacts_new, t, self.b, kappa, n=n_ee, ws=self._ws_ee)
            if n_pt:
                self._ws_pt = hessian_workspace(self.contacts_pt, getattr(self, "_ws_pt", None))
                contact_hessian_pt(states, self.soup, self.contacts_pt, t, self.b, n_ee, kappa, n=n_pt,
                                   ws=self._ws_pt)
            if not build_bsr:
                return None
            prev = getattr(self, "collision_hessian", None)
            H, status = contact_bsr(self.contacts_new, n_ee, self.contacts_pt, n_pt, self.soup.n_verts, t, out=prev)
            if status & 4:  # a row with too many distinct columns: generic assembly
                H = bsr_from_triplets(self.soup.n_verts, self.soup.n_verts, t.rows, t.cols, t.vals, count=nnz,
                                      out=H)
            self.collision_hessian = H
        return self.collision_hessian

    def compute_collision_energy(self, detect: bool = True) -> float:
        """dynamic_contacts.py:299-308: detect, sum the barrier energy
        (double), return it times h^2."""
        if detect:
            with self.profile_timer("collision energy detect"):
                self.detect_collision()
        e = torch.zeros(1, dtype=torch.float64, device=self.device)
        kappa = float(self.contact_stiffness)
        states = getattr(self, "states", None)
        if self.n_contacts:
            contact_energy_ee(states, self.soup, self.contacts_new, e, kappa, n=self.n_contacts)
        if self.n_contacts_pt:
            contact_energy_pt(states, self.soup, self.contacts_pt, e, kappa, n=self.n_contacts_pt)
        return float(e.item()) * self.h * self.h
