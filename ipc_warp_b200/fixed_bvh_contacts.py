"""Contact solver whose DCD broad phase uses immutable body-local hierarchies:
the ``FixedBodyContactSolver`` of the reference (fixed_bvh_contacts.py:503-827),
backed by ipcb_body_pairs / ipcb_fixed_dcd_* / ipcb_fixed_*_toi.

``soup.xcs`` holds body-local rest coordinates and ``affine_q`` four vec3 per
body, ``[p, A[:,0], A[:,1], A[:,2]]`` (x = p + A r).  The hierarchies of every
body's rest edges and triangles are built once; a query primitive of body a
is mapped into body b's frame and tested against b's hierarchy, and accepted
by the same exact world-space predicate as the dynamic path, so the candidate
sets equal the dynamic DCD's with same-body pairs excluded.  CCD queries the
same hierarchies with swept local boxes inflated by the target frame's
motion; a near-singular body (|det A| < 1e-8 at either end of the step)
falls back to the inherited swept-hierarchy CCD as in the reference, and to
the inherited DCD with same-body pairs excluded (where the reference would
invert the singular frame).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as N
from . import contact as contact_mod
from .contact import ContactSolverBase
from .lbvh import Bvh

STATUS_SINGULAR = 32


class FixedBodyContactSolver(ContactSolverBase):
    """fixed_bvh_contacts.py:503-827 (mixin; requires ``self.soup``)."""

    def initialize_fixed_body_bvhs(self, affine_q: torch.Tensor):
        """fixed_bvh_contacts.py:511-603: per-body rest hierarchies."""
        self.affine_q = affine_q
        soup = self.soup
        dev = soup.xcs.device
        rest = soup.xcs.double().cpu().numpy()
        body = soup.body.cpu().numpy().astype(np.int64)
        edges = soup.edges.cpu().numpy().reshape(-1, 2)
        tris = soup.triangles.cpu().numpy().reshape(-1, 3)
        if not hasattr(self, "n_bodies"):
            self.n_bodies = int(body.max()) + 1
        nb = self.n_bodies
        lo = np.zeros((nb, 3), np.float32)
        hi = np.zeros((nb, 3), np.float32)
        vids, eids, tids = [], [], []
        self._fixed_bvhs = []
        ew, tw = [], []
        for b in range(nb):
            v = np.flatnonzero(body == b).astype(np.int32)
            e = np.flatnonzero(body[edges[:, 0]] == b).astype(np.int32) if len(edges) else np.zeros(0, np.int32)
            t = np.flatnonzero(body[tris[:, 0]] == b).astype(np.int32) if len(tris) else np.zeros(0, np.int32)
            vids.append(v)
            eids.append(e)
            tids.append(t)
            if len(v):
                lo[b] = rest[v].min(axis=0)
                hi[b] = rest[v].max(axis=0)
            for ids, prim, out in ((e, edges, ew), (t, tris, tw)):
                if len(ids) == 0:
                    out.append(0)
                    continue
                pts = rest[prim[ids]]
                blo = torch.tensor(pts.min(axis=1).astype(np.float32), device=dev)
                bhi = torch.tensor(pts.max(axis=1).astype(np.float32), device=dev)
                bvh = Bvh(blo, bhi)
                self._fixed_bvhs.append((bvh, blo, bhi))
                out.append(bvh.c.wide)

        def flat(lists):
            counts = np.array([len(a) for a in lists], np.int64)
            off = np.zeros(nb + 1, np.int32)
            off[1:] = np.cumsum(counts)
            vals = np.concatenate(lists).astype(np.int32) if off[-1] else np.zeros(1, np.int32)
            return (torch.tensor(off, device=dev), torch.tensor(vals, device=dev), int(counts.max(initial=0)))

        i32 = dict(dtype=torch.int32, device=dev)
        self.fixed_vertex_offsets, self.fixed_vertex_ids_flat, self.fixed_max_vertices = flat(vids)
        self.fixed_edge_offsets, self.fixed_edge_ids_flat, self.fixed_max_edges = flat(eids)
        self.fixed_triangle_offsets, self.fixed_triangle_ids_flat, self.fixed_max_triangles = flat(tids)
        self.fixed_edge_bvh_ids = torch.tensor(ew, dtype=torch.int64, device=dev)
        self.fixed_triangle_bvh_ids = torch.tensor(tw, dtype=torch.int64, device=dev)
        self.fixed_local_lower = torch.tensor(lo, device=dev)
        self.fixed_local_upper = torch.tensor(hi, device=dev)
        self._frames = torch.zeros(19 * nb, dtype=torch.float64, device=dev)
        self._motion = torch.zeros(3 * nb, dtype=torch.float64, device=dev)
        cap = max(nb * (nb - 1) // 2, 1)
        self.fixed_body_pairs = torch.zeros((cap, 2), **i32)
        self.fixed_body_pair_count = torch.zeros(1, **i32)
        self._fixed_status = torch.zeros(1, **i32)
        # the reference's mode switches; one implementation serves all modes
        self.fixed_pair_cull_mode = "kernel"
        self.fixed_query_mode = "scalar"
        self.tile_query_threads = 32
        if hasattr(self, "abd_fixed"):
            self.fixed_body_flags = self.abd_fixed
        else:
            self.fixed_body_flags = torch.zeros(nb, **i32)
        self._bodies = N.Bodies(nb, N.ptr(self.fixed_local_lower), N.ptr(self.fixed_local_upper),
                                N.ptr(self.fixed_edge_offsets), N.ptr(self.fixed_edge_ids_flat),
                                N.ptr(self.fixed_triangle_offsets), N.ptr(self.fixed_triangle_ids_flat),
                                N.ptr(self.fixed_vertex_offsets), N.ptr(self.fixed_vertex_ids_flat),
                                N.ptr(self.fixed_edge_bvh_ids), N.ptr(self.fixed_triangle_bvh_ids),
                                self.fixed_max_edges, self.fixed_max_triangles, self.fixed_max_vertices,
                                N.ptr(self._frames), N.ptr(self._motion))
        self._ccd_ws_fixed = torch.empty(N.size("ipcb_toi_workspace", max(1 << 20, 4 * soup.n_edges)),
                                         dtype=torch.uint8, device=dev)

    def _read(self, *tensors):
        out = torch.cat([t.reshape(-1).to(torch.int64) for t in tensors]).cpu()
        return [int(v) for v in out]

    def _pairs(self, swept_dq=None):
        """(n_pairs, singular) after the (swept) body cull."""
        q = self.affine_q
        fp64 = int(q.dtype == torch.float64)
        while True:
            self.fixed_body_pair_count.zero_()
            self._fixed_status.zero_()
            cap = self.fixed_body_pairs.shape[0]
            if swept_dq is None:
                N.call("ipcb_body_pairs", ctypes.byref(self._bodies), fp64, N.ptr(q),
                       float(2.0 * contact_mod._thickness), N.ptr(self.fixed_body_pairs), cap,
                       N.ptr(self.fixed_body_pair_count), N.ptr(self._fixed_status), N.stream_handle())
            else:
                N.call("ipcb_body_pairs_swept", ctypes.byref(self._bodies), fp64, N.ptr(q), N.ptr(swept_dq), 1.0e-7,
                       N.ptr(self.fixed_body_pairs), cap, N.ptr(self.fixed_body_pair_count),
                       N.ptr(self._fixed_status), N.stream_handle())
            n, st = self._read(self.fixed_body_pair_count, self._fixed_status)
            if n <= cap:
                return n, bool(st & STATUS_SINGULAR)
            self.fixed_body_pairs = torch.zeros((1 << (n - 1).bit_length(), 2), dtype=torch.int32,
                                                device=q.device)

    def detect_collision(self):
        """fixed_bvh_contacts.py:777-827."""
        self.compute_V(ret=False)
        self._pack()
        n_pairs, singular = self._pairs()
        if singular:
            # a near-singular frame has no usable inverse: the swept-hierarchy
            # query with same-body pairs excluded gives the same contact set
            keep = self.disable_self_collision
            self.disable_self_collision = True
            try:
                return ContactSolverBase.detect_collision(self)
            finally:
                self.disable_self_collision = keep
        soup = self.soup.c_struct()
        s = N.stream_handle()
        th = float(contact_mod._thickness)
        while True:
            self.contacts_new.cnt.zero_()
            self.contacts_pt.cnt.zero_()
            self._status.zero_()
            if n_pairs:
                N.call("ipcb_fixed_dcd_ee", ctypes.byref(soup), N.ptr(self.x4), ctypes.byref(self._bodies),
                       N.ptr(self.fixed_body_pairs), n_pairs, th, ctypes.byref(self.contacts_new.c_struct()),
                       N.ptr(self._status), s)
                N.call("ipcb_fixed_dcd_pt", ctypes.byref(soup), N.ptr(self.x4), ctypes.byref(self._bodies),
                       N.ptr(self.fixed_body_pairs), n_pairs, th, ctypes.byref(self.contacts_pt.c_struct()),
                       N.ptr(self._status), s)
            n_ee, n_pt = self._read_counts()
            grown = False
            if n_ee > self.contacts_new.capacity:
                self._grow_contact_list(self.contacts_new, n_ee)
                grown = True
            if n_pt > self.contacts_pt.capacity:
                self._grow_contact_list(self.contacts_pt, n_pt, point_triangle=True)
                grown = True
            if not grown:
                break
        self.n_contacts, self.n_contacts_pt = n_ee, n_pt
        self.fixed_body_pair_count_host = n_pairs

    def collision_free_step(self, dx: torch.Tensor) -> float:
        """fixed_bvh_contacts.py:719-775: fixed-hierarchy CCD when the affine
        step ``self.abd_states.dx`` is known, else the swept-hierarchy path."""
        abd = getattr(self, "abd_states", None)
        if abd is None:
            return ContactSolverBase.collision_free_step(self, dx)
        soup = self.soup.c_struct()
        s = N.stream_handle()
        N.call("ipcb_add_dx", ctypes.byref(soup), N.ptr(dx), N.ptr(self.ccd_x1), s)
        n_pairs, singular = self._pairs(abd.dx)
        if singular:
            return ContactSolverBase.collision_free_step(self, dx)
        self.ccd_toi.fill_(1.0)
        self._status.zero_()
        if n_pairs:
            ws = self._ccd_ws_fixed
            N.call("ipcb_fixed_edge_edge_toi", ctypes.byref(soup), N.ptr(self.ccd_x1), ctypes.byref(self._bodies),
                   N.ptr(self.fixed_body_flags), N.ptr(self.fixed_body_pairs), n_pairs, 1.0e-7, N.ptr(self.ccd_toi),
                   N.ptr(self._status), N.ptr(ws), ws.numel(), s)
            N.call("ipcb_fixed_point_triangle_toi", ctypes.byref(soup), N.ptr(self.ccd_x1),
                   ctypes.byref(self._bodies), N.ptr(self.fixed_body_pairs), n_pairs, 1.0e-7, N.ptr(self.ccd_toi),
                   N.ptr(self._status), N.ptr(ws), ws.numel(), s)
        return self._step_bound()
