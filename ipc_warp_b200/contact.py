"""Drop-in contact solver base: the Python surface of contact.py (reference
contact.py:444-750) backed by the sm_100a kernels of libipcb200.

A class that mixes in :class:`ContactSolverBase` sets ``self.soup`` (a
:class:`Soup`) before calling ``ContactSolverBase.__init__(self)``, exactly as
with the reference mixin.  Afterwards it has the reference attributes
``bvh_edges``, ``tri_mesh``, ``ccd_edge_bvh``, ``ccd_triangle_bvh``,
``ccd_toi``, ``ccd_x1``, ``contacts_new``, ``contacts_pt``, ``n_contacts``,
``n_contacts_pt``, ``disable_self_collision`` and the methods
``detect_collision()``, ``collision_free_step(dx)``, ``update_bvh()``,
``compute_edge_aabbs()``, ``compute_V()`` and ``_grow_contact_list()``.

Module globals mirror contact.py:14-22 (``_thickness``, ``buffer``,
``contact_volume``, ``disable_self_collision``, ``verbose``); they are read
at call time, so a scene sets ``contact._thickness = dhat / 2`` as with the
reference (dhat = l0 = 2 * _thickness, contact.py:180).
"""
from __future__ import annotations

import ctypes
import warnings
from contextlib import nullcontext
from dataclasses import dataclass

import torch

from . import _native as N
from . import scalar_types as st
from .lbvh import Bvh

_thickness = 0.01
contact_volume = 10000
buffer = _thickness
eps = 1e-6
disable_self_collision = False
verbose = False

# IPCB_STATUS_STACK | IPCB_STATUS_ROOT_ITERS: a query that ran out of its
# traversal stack, its visit bound or its root iterations may have missed an
# impact, so its TOI is no bound
QUERY_FAILED = 1 | 2


@dataclass
class Soup:
    """fem/geometry.py:165-171.  Positions are (V, 3) tensors of the scalar
    type, index arrays flat int32 like the reference."""
    xcs: torch.Tensor
    triangles: torch.Tensor
    edges: torch.Tensor
    body: torch.Tensor
    x_transformed: torch.Tensor

    @property
    def n_verts(self) -> int:
        return self.xcs.shape[0]

    @property
    def n_edges(self) -> int:
        return self.edges.shape[0] // 2

    @property
    def n_tris(self) -> int:
        return self.triangles.shape[0] // 3

    def c_struct(self, x: torch.Tensor | None = None) -> N.Soup:
        x = self.x_transformed if x is None else x
        if x.dtype not in (torch.float32, torch.float64) or not x.is_contiguous():
            raise ValueError("positions must be contiguous float32/float64 (V, 3)")
        if self.xcs.dtype != x.dtype:
            raise ValueError("xcs and x_transformed must share the scalar type")
        return N.Soup(self.n_verts, self.n_edges, self.n_tris, int(x.dtype == torch.float64), N.ptr(x),
                      N.ptr(self.xcs), N.ptr(self.edges), N.ptr(self.triangles), N.ptr(self.body))

    @staticmethod
    def from_numpy(x, edges, triangles, body, xcs=None, device="cuda", dtype=None) -> "Soup":
        dtype = dtype or st.scalar()
        xt = torch.as_tensor(x, dtype=dtype, device=device).contiguous()
        xr = xt.clone() if xcs is None else torch.as_tensor(xcs, dtype=dtype, device=device).contiguous()
        i32 = lambda a: torch.as_tensor(a, dtype=torch.int32, device=device).reshape(-1).contiguous()
        return Soup(xcs=xr, triangles=i32(triangles), edges=i32(edges), body=i32(body), x_transformed=xt)


class Contacts:
    """contact.py:61-80 ``Contacts`` with its ``XConstraint`` records stored
    as columns: ``a1a2b1b2`` int32 (cap, 4), ``e0e1`` int32 (cap, 2), ``l0``,
    ``alpha``, ``lam`` scalar (cap,), ``cnt`` int32 (1,).  ``htable`` is
    allocated for attribute compatibility; the reference writes it without
    ever reading it (contact.py:183), so it is left at -1."""

    def __init__(self, capacity: int, dtype: torch.dtype, device):
        self.capacity = int(capacity)
        self.dtype = dtype
        self.device = device
        self.a1a2b1b2 = torch.zeros((self.capacity, 4), dtype=torch.int32, device=device)
        self.e0e1 = torch.zeros((self.capacity, 2), dtype=torch.int32, device=device)
        self.l0 = torch.zeros(self.capacity, dtype=dtype, device=device)
        self.alpha = torch.zeros(self.capacity, dtype=dtype, device=device)
        self.lam = torch.zeros(self.capacity, dtype=dtype, device=device)
        self.cnt = torch.zeros(1, dtype=torch.int32, device=device)
        self.htable = torch.full((8191,), -1, dtype=torch.int32, device=device)

    @property
    def list(self) -> "Contacts":
        return self

    def c_struct(self) -> N.Contacts:
        return N.Contacts(N.ptr(self.a1a2b1b2), N.ptr(self.e0e1), N.ptr(self.l0), N.ptr(self.alpha),
                          N.ptr(self.lam), N.ptr(self.cnt), self.capacity)

    def grow(self, capacity: int) -> None:
        self.__init__(capacity, self.dtype, self.device)

    def records(self, n: int) -> torch.Tensor:
        """(n, 6) int32 [a1, a2, b1, b2, e0, e1] of the first n records."""
        return torch.cat([self.a1a2b1b2[:n], self.e0e1[:n]], dim=1)


def _next_pow2(n: int) -> int:
    return 1 << (max(n, 1) - 1).bit_length()


class ContactSolverBase:
    """contact.py:444-750 mixin.  Requires ``self.soup``."""

    def __init__(self):
        soup: Soup = self.soup
        self.disable_self_collision = disable_self_collision
        dev = soup.xcs.device
        self.device = dev
        dtype = soup.xcs.dtype
        n_edges, n_nodes, n_tris = soup.n_edges, soup.n_verts, soup.n_tris
        f32 = dict(dtype=torch.float32, device=dev)
        self.x4 = torch.zeros((n_nodes, 4), **f32)  # float32 mesh copy (contact.py:476, x_mesh)
        self.bvh_edges_lower = torch.zeros((n_edges, 3), **f32)
        self.bvh_edges_upper = torch.zeros((n_edges, 3), **f32)
        self.compute_edge_aabbs()
        self.bvh_edges = Bvh(self.bvh_edges_lower, self.bvh_edges_upper)
        # CCD boxes are refit into the DCD hierarchies (same primitives, same
        # topology); detect_collision refits them back before every query.
        self.ccd_edge_lower = torch.zeros((n_edges, 3), **f32)
        self.ccd_edge_upper = torch.zeros((n_edges, 3), **f32)
        self.ccd_edge_bvh = self.bvh_edges
        self.ccd_toi = torch.ones(1, dtype=dtype, device=dev)
        self.ccd_x1 = torch.zeros_like(soup.x_transformed)
        self.has_triangles = n_tris > 0
        if self.has_triangles:
            self.tri_lower = torch.zeros((n_tris, 3), **f32)
            self.tri_upper = torch.zeros((n_tris, 3), **f32)
            self._triangle_aabbs()
            self.tri_mesh = Bvh(self.tri_lower, self.tri_upper)
            self.ccd_triangle_lower = torch.zeros((n_tris, 3), **f32)
            self.ccd_triangle_upper = torch.zeros((n_tris, 3), **f32)
            self.ccd_triangle_bvh = self.tri_mesh
        self.contacts_new = Contacts(contact_volume, dtype, dev)
        self.contacts_pt = Contacts(contact_volume, dtype, dev)
        self.contacts_list_new = self.contacts_new
        self.contacts_list_pt = self.contacts_pt
        self.n_contacts = 0
        self.n_contacts_pt = 0
        self._status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.query_status = 0  # status word of the last detect_collision / collision_free_step
        self.ccd_refusals = 0  # collision_free_step calls refused for a failed query
        # CCD candidate staging (a query that overflows it is redone inline)
        cap = max(1 << 20, 4 * max(n_edges, n_nodes))
        self._toi_ws = torch.empty(N.size("ipcb_toi_workspace", cap), dtype=torch.uint8, device=dev)
        self._counts_host = torch.zeros(3, dtype=torch.int32).pin_memory() if dev.type == "cuda" else None

    # --------------------------------------------------------------- hooks
    def profile_timer(self, name):
        return nullcontext()

    def compute_V(self, ret=True):
        return None

    # --------------------------------------------------------------- boxes
    def _pack(self):
        N.call("ipcb_pack_positions", ctypes.byref(self.soup.c_struct()), N.ptr(self.x4), N.stream_handle())

    def compute_edge_aabbs(self):
        """contact.py:679-681: edge boxes padded by _thickness + buffer."""
        self._pack()
        N.call("ipcb_edge_aabbs", ctypes.byref(self.soup.c_struct()), N.ptr(self.x4), float(_thickness + buffer),
               N.ptr(self.bvh_edges_lower), N.ptr(self.bvh_edges_upper), N.stream_handle())

    def _triangle_aabbs(self):
        N.call("ipcb_triangle_aabbs", ctypes.byref(self.soup.c_struct()), N.ptr(self.x4), 0.0,
               N.ptr(self.tri_lower), N.ptr(self.tri_upper), N.stream_handle())

    def update_bvh(self):
        """contact.py:672-677: edge boxes + refit, float32 mesh copy + refit.
        With ``bvh_rebuild_interval`` = k > 0 the hierarchies are rebuilt
        (new Morton order) every k-th call instead of refit."""
        self.compute_edge_aabbs()
        k = getattr(self, "bvh_rebuild_interval", 0)
        self._bvh_calls = getattr(self, "_bvh_calls", 0) + 1
        rebuild = k > 0 and self._bvh_calls % k == 0
        if rebuild:
            self.bvh_edges.rebuild()
        else:
            self.bvh_edges.refit()
        if self.has_triangles:
            self._triangle_aabbs()
            if rebuild:
                self.tri_mesh.rebuild()
            else:
                self.tri_mesh.refit()

    # ----------------------------------------------------------------- DCD
    def _grow_contact_list(self, contacts: Contacts, required: int, point_triangle: bool = False):
        """contact.py:523-537: grow to the next power of two."""
        contacts.grow(_next_pow2(required))
        if point_triangle:
            self.contacts_list_pt = contacts
        else:
            self.contacts_list_new = contacts
        if verbose:
            print(f"contact buffer grown to {contacts.capacity}")

    def _launch_dcd(self, which: str):
        soup = self.soup.c_struct()
        s = N.stream_handle()
        if which == "ee":
            self.contacts_new.cnt.zero_()
            N.call("ipcb_dcd_ee", ctypes.byref(soup), N.ptr(self.x4), ctypes.byref(self.bvh_edges.c),
                   float(_thickness), float(_thickness + buffer), int(self.disable_self_collision),
                   ctypes.byref(self.contacts_new.c_struct()), N.ptr(self._status), s)
        else:
            self.contacts_pt.cnt.zero_()
            N.call("ipcb_dcd_pt", ctypes.byref(soup), N.ptr(self.x4), ctypes.byref(self.tri_mesh.c),
                   float(_thickness), float(2.0 * (_thickness + buffer)), int(self.disable_self_collision), None,
                   ctypes.byref(self.contacts_pt.c_struct()), N.ptr(self._status), s)

    def _read_counts(self):
        """One host read of both list counts and the query status word (kept
        in ``query_status``)."""
        h = self._counts_host
        h[0:1].copy_(self.contacts_new.cnt, non_blocking=True)
        if self.has_triangles:
            h[1:2].copy_(self.contacts_pt.cnt, non_blocking=True)
        else:
            h[1] = 0
        h[2:3].copy_(self._status, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        self.query_status = int(h[2])
        return int(h[0]), int(h[1])

    def detect_collision(self):
        """contact.py:687-725.  Both queries are launched before the single
        count read; an overflowed list is grown and its query relaunched."""
        self.compute_V(ret=False)
        self._status.zero_()
        with self.profile_timer("collision BVH refit"):
            self.update_bvh()
        with self.profile_timer("EE collision query"):
            self._launch_dcd("ee")
        if self.has_triangles:
            with self.profile_timer("PT collision query"):
                self._launch_dcd("pt")
        with self.profile_timer("contact count host transfer"):
            n_ee, n_pt = self._read_counts()
        relaunched = False
        if n_ee > self.contacts_new.capacity:
            self._grow_contact_list(self.contacts_new, n_ee)
            self._launch_dcd("ee")
            relaunched = True
        if n_pt > self.contacts_pt.capacity:
            self._grow_contact_list(self.contacts_pt, n_pt, point_triangle=True)
            self._launch_dcd("pt")
            relaunched = True
        if relaunched:
            n_ee, n_pt = self._read_counts()
        self.n_contacts, self.n_contacts_pt = n_ee, (n_pt if self.has_triangles else 0)
        if self.query_status & QUERY_FAILED:
            warnings.warn(f"contact query ran out of its traversal bound (status {self.query_status}): "
                          "the candidate lists may be incomplete", RuntimeWarning, stacklevel=2)
        if verbose:
            print(f"n ee contacts = {self.n_contacts}\nn pt contacts = {self.n_contacts_pt}")

    # ----------------------------------------------------------------- CCD
    def collision_free_step(self, dx: torch.Tensor) -> float:
        """contact.py:539-585: conservative CCD bound for x -= alpha * dx;
        returns 0.9 * toi if toi < 1 else 1."""
        self._launch_ccd(dx)
        return self._step_bound()

    def _step_bound(self) -> float:
        """One host read of the TOI and the query status.  The bound is
        0.9 * toi (1 when nothing collides), or 0 -- no step -- when a query
        set IPCB_STATUS_STACK or IPCB_STATUS_ROOT_ITERS: such a query may have
        missed an earlier impact, so its TOI is no bound.  Refusals are
        counted in ``ccd_refusals``."""
        toi, status = torch.cat([self.ccd_toi.double(), self._status.double()]).tolist()
        return self._bound_from(toi, int(status))

    def _bound_from(self, toi: float, status: int) -> float:
        self.query_status = status
        if status & QUERY_FAILED:
            self.ccd_refusals += 1
            return 0.0
        return 0.9 * toi if toi < 1.0 else 1.0

    def _launch_ccd(self, dx: torch.Tensor, reset_status: bool = True):
        """The CCD queries of collision_free_step; the TOI stays in ccd_toi
        and the queries' status bits in _status (zeroed first unless
        reset_status is False)."""
        soup = self.soup.c_struct()
        s = N.stream_handle()
        pad = 1e-7
        N.call("ipcb_add_dx", ctypes.byref(soup), N.ptr(dx), N.ptr(self.ccd_x1), s)
        N.call("ipcb_swept_edge_aabbs", ctypes.byref(soup), N.ptr(self.ccd_x1), pad, N.ptr(self.ccd_edge_lower),
               N.ptr(self.ccd_edge_upper), s)
        self.ccd_edge_bvh.refit(self.ccd_edge_lower, self.ccd_edge_upper)
        self.ccd_toi.fill_(1.0)
        if reset_status:
            self._status.zero_()
        N.call("ipcb_edge_edge_toi", ctypes.byref(soup), N.ptr(self.ccd_x1), ctypes.byref(self.ccd_edge_bvh.c),
               N.ptr(self.ccd_edge_lower), N.ptr(self.ccd_edge_upper), int(self.disable_self_collision),
               N.ptr(self.ccd_toi), N.ptr(self._status), N.ptr(self._toi_ws), self._toi_ws.numel(), s)
        if self.has_triangles:
            N.call("ipcb_swept_triangle_aabbs", ctypes.byref(soup), N.ptr(self.ccd_x1), pad,
                   N.ptr(self.ccd_triangle_lower), N.ptr(self.ccd_triangle_upper), s)
            self.ccd_triangle_bvh.refit(self.ccd_triangle_lower, self.ccd_triangle_upper)
            N.call("ipcb_point_triangle_toi", ctypes.byref(soup), N.ptr(self.ccd_x1),
                   ctypes.byref(self.ccd_triangle_bvh.c), pad, int(self.disable_self_collision),
                   N.ptr(self.ccd_toi), N.ptr(self._status), N.ptr(self._toi_ws), self._toi_ws.numel(), s)

    def new_intersections(self, x0: torch.Tensor, x1: torch.Tensor) -> float:
        """contact.py:587-670 (the augmented-Lagrangian solver's CCD): every
        EE / PT pair that collides on the straight path x0 -> x1 becomes a
        record of ``contacts_new`` / ``contacts_pt`` (alpha = its time of
        impact); returns 0.9 * toi if toi < 1 else 1.  Lists grow and the
        query reruns when they overflow, as the reference."""
        soup = self.soup.c_struct(x0)
        s = N.stream_handle()
        pad = 1e-7
        th = float(_thickness)
        excl = int(self.disable_self_collision)
        N.call("ipcb_swept_edge_aabbs", ctypes.byref(soup), N.ptr(x1), pad, N.ptr(self.ccd_edge_lower),
               N.ptr(self.ccd_edge_upper), s)
        self.ccd_edge_bvh.refit(self.ccd_edge_lower, self.ccd_edge_upper)
        self._status.zero_()

        def edges():
            self.contacts_new.cnt.zero_()
            self.ccd_toi.fill_(1.0)
            N.call("ipcb_edge_edge_intersections", ctypes.byref(soup), N.ptr(x1), ctypes.byref(self.ccd_edge_bvh.c),
                   N.ptr(self.ccd_edge_lower), N.ptr(self.ccd_edge_upper), excl, th, N.ptr(self.ccd_toi),
                   ctypes.byref(self.contacts_new.c_struct()), N.ptr(self._status), N.ptr(self._toi_ws),
                   self._toi_ws.numel(), s)
            return int(self.contacts_new.cnt.item())

        n = edges()
        if n > self.contacts_new.capacity:
            self._grow_contact_list(self.contacts_new, n)
            n = edges()
        self.n_contacts = n
        if self.has_triangles:
            N.call("ipcb_swept_triangle_aabbs", ctypes.byref(soup), N.ptr(x1), pad, N.ptr(self.ccd_triangle_lower),
                   N.ptr(self.ccd_triangle_upper), s)
            self.ccd_triangle_bvh.refit(self.ccd_triangle_lower, self.ccd_triangle_upper)

            def points():
                self.contacts_pt.cnt.zero_()
                N.call("ipcb_point_triangle_intersections", ctypes.byref(soup), N.ptr(x1),
                       ctypes.byref(self.ccd_triangle_bvh.c), pad, excl, th, N.ptr(self.ccd_toi),
                       ctypes.byref(self.contacts_pt.c_struct()), N.ptr(self._status), N.ptr(self._toi_ws),
                       self._toi_ws.numel(), s)
                return int(self.contacts_pt.cnt.item())

            n = points()
            if n > self.contacts_pt.capacity:
                self._grow_contact_list(self.contacts_pt, n, point_triangle=True)
                n = points()
            self.n_contacts_pt = n
        else:
            self.n_contacts_pt = 0
        return self._step_bound()

    def edge_triangle_crossings(self, capacity: int = 0):
        """Intersection check of the current positions: the number of
        (surface edge, surface triangle) pairs, without a shared vertex, whose
        segment crosses the triangle (an accepted IPC step leaves none), and
        up to ``capacity`` of them as an (m, 2) int32 tensor (edge,
        triangle).  Refits the triangle hierarchy to the positions (the next
        detect_collision refits it again)."""
        if not self.has_triangles:
            return 0, torch.zeros((0, 2), dtype=torch.int32, device=self.device)
        self._pack()
        self._triangle_aabbs()
        self.tri_mesh.refit()
        count = torch.zeros(1, dtype=torch.int32, device=self.device)
        pairs = torch.zeros((max(capacity, 1), 2), dtype=torch.int32, device=self.device)
        st = torch.zeros(1, dtype=torch.int32, device=self.device)
        N.call("ipcb_edge_triangle_crossings", ctypes.byref(self.soup.c_struct()), ctypes.byref(self.tri_mesh.c),
               N.ptr(count), N.ptr(pairs), int(capacity), N.ptr(st), N.stream_handle())
        n, status = (int(v) for v in torch.cat([count, st]).tolist())
        if status & QUERY_FAILED:
            raise RuntimeError(f"intersection check ran out of its traversal bound (status {status})")
        return n, pairs[:min(n, capacity)]

    @property
    def status(self) -> int:
        """OR of IPCB_STATUS_* bits raised by the last queries."""
        return int(self._status.item())
