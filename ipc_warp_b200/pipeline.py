"""The per-Newton-iteration contact pipeline as one object.

``ContactPipeline`` is a ready-made host for :class:`ContactBarrierMixin`:
it owns the soup, the force accumulator ``b`` and the step ``h``, and
``iteration(dx)`` runs what RodComplexBC does for contact in one Newton
iteration (dynamic_contacts.py:272-308 with contact.py:539-725):

  1. ``detect_collision()``          BVH refit, EE and PT candidate lists
  2. ``compute_contact_hessian()``   16 triplets per record, force into b,
                                     canonical BSR of the contact Hessian
  3. ``compute_collision_energy()``  barrier energy (double) x h^2
  4. ``collision_free_step(dx)``     CCD step bound for x -= alpha dx
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from . import contact
from .contact import Soup
from .bsr import Triplets, contact_bsr
from .dynamic_contacts import (ContactBarrierMixin, contact_energy_ee, contact_energy_pt, contact_hessian_ee,
                               contact_hessian_pt_after, hessian_workspace)


@dataclass
class NewtonState:
    """fem/params.py:43-50 (the fields the contact pipeline touches)."""
    x: torch.Tensor
    dx: torch.Tensor


@dataclass
class IterationResult:
    n_ee: int
    n_pt: int
    energy: float
    alpha: float
    status: int = 0  # IPCB_STATUS_* bits of the queries; a failed query gives alpha = 0


class ContactPipeline(ContactBarrierMixin):
    def __init__(self, soup: Soup, dhat: float, kappa: float, h: float = 1e-2, exclude_same_body: bool = False):
        contact._thickness = 0.5 * dhat
        contact.buffer = 0.5 * dhat
        self.soup = soup
        self.h = float(h)
        self.contact_stiffness = float(kappa)
        self.states = NewtonState(x=soup.x_transformed, dx=torch.zeros_like(soup.x_transformed))
        self.b = torch.zeros_like(soup.x_transformed)
        ContactBarrierMixin.__init__(self)
        self.disable_self_collision = exclude_same_body
        self.collision_triplets = None
        self.collision_hessian = None
        dev = soup.x_transformed.device
        self._bsr_status = torch.zeros(1, dtype=torch.int32, device=dev)
        self._energy = torch.zeros(1, dtype=torch.float64, device=dev)
        pin = dev.type == "cuda"
        self.use_graph = True
        self._graph = None
        if pin:
            self._side = torch.cuda.Stream(device=dev)
            self._ccd_e = torch.cuda.Stream(device=dev)
            self._ccd_t = torch.cuda.Stream(device=dev)
            self._copy_in = torch.cuda.Stream(device=dev)
            self._copy_out = torch.cuda.Stream(device=dev)
            self._x1_done = torch.cuda.Event()
            self._ee_done = torch.cuda.Event()
            self._pt_done = torch.cuda.Event()
            self._toi_ws_pt = torch.empty_like(self._toi_ws)
        self._dx_buf = torch.zeros_like(soup.x_transformed)
        self._host_io = None  # (x, dx, b) pinned host tensors during iteration_host
        self._last_stepwise = False
        self._readback = {"counts": torch.zeros(4, dtype=torch.int32, pin_memory=pin),
                          "energy": torch.zeros(1, dtype=torch.float64, pin_memory=pin),
                          "toi": torch.zeros(1, dtype=soup.x_transformed.dtype, pin_memory=pin)}

    @classmethod
    def from_scene(cls, scene, dtype=None, device="cuda", exclude_same_body=False) -> "ContactPipeline":
        soup = Soup.from_numpy(scene.x, scene.edges, scene.triangles, scene.body, xcs=scene.xcs, device=device,
                               dtype=dtype)
        return cls(soup, scene.dhat, scene.kappa, exclude_same_body=exclude_same_body)

    def iteration(self, dx: torch.Tensor | None = None) -> IterationResult:
        """One Newton iteration's contact work.  On a GPU every stage is
        enqueued without a host read (list counts taken on the device, PT
        records placed after the EE count, the contact BSR sized for the
        list capacities) and the counts, the BSR status, the energy and the
        TOI come back in one read at the end.  After one such iteration the
        whole sequence is captured in a CUDA graph and replayed (recaptured
        when a buffer is reallocated).  A list that overflowed or a BSR row
        with too many columns sends the iteration through the step-by-step
        calls, which grow the lists and pick the generic assembly."""
        if dx is not None:
            self.states.dx = dx
        if self.device.type != "cuda":
            return self.iteration_stepwise()
        if self._dx_buf.data_ptr() != self.states.dx.data_ptr():
            self._dx_buf.copy_(self.states.dx)
        key = self._graph_key()
        if self.use_graph and self._graph is not None and self._graph[0] == key:
            self._graph[1].replay()
        else:
            self._enqueue()
        torch.cuda.current_stream().synchronize()
        h = self._readback
        ee, pt = self.contacts_new, self.contacts_pt
        n_ee, n_pt, st, qst = (int(v) for v in h["counts"])
        self._last_stepwise = False
        if n_ee > ee.capacity or n_pt > pt.capacity or st & 4:
            self._graph = None
            self._last_stepwise = True
            return self.iteration_stepwise()
        if self.use_graph and (self._graph is None or self._graph[0] != key):
            self._capture(self._graph_key())  # the eager pass may have (re)allocated buffers
        self.n_contacts, self.n_contacts_pt = n_ee, n_pt
        alpha = self._bound_from(float(h["toi"][0]), qst)
        return IterationResult(n_ee, n_pt, float(h["energy"][0]) * self.h * self.h, alpha, qst)

    def _graph_key(self):
        ee, pt, t, H = self.contacts_new, self.contacts_pt, self.collision_triplets, self.collision_hessian
        ws = tuple(None if getattr(self, a, None) is None else getattr(self, a).data_ptr()
                   for a in ("_ws_ee", "_ws_pt"))
        io = None if self._host_io is None else tuple(a.data_ptr() for a in self._host_io)
        return (ee.a1a2b1b2.data_ptr(), ee.capacity, pt.a1a2b1b2.data_ptr(), pt.capacity,
                None if t is None else t.rows.data_ptr(), None if H is None else H.values.data_ptr(),
                None if H is None else H._ws.data_ptr(), ws, io, getattr(self, "bvh_rebuild_interval", 0))

    def iteration_host(self, x: torch.Tensor, dx: torch.Tensor, b: torch.Tensor) -> IterationResult:
        """iteration() from host memory: positions x and direction dx (V, 3)
        copied in, the contact force b copied out (pinned tensors of the
        soup's dtype).  On a GPU the copies are part of the enqueued (and
        graph-replayed) sequence: x first, dx on its own stream beside the
        discrete queries (only the CCD reads it), and b as soon as the narrow
        phase has written it, beside the BSR, energy and CCD stages."""
        if self.device.type != "cuda":
            self.soup.x_transformed.copy_(x)
            res = self.iteration(dx.to(self.device))
            b.copy_(self.b)
            return res
        self._host_io = (x, dx, b)
        self.states.dx = self._dx_buf  # filled by the copy in the sequence
        try:
            res = self.iteration()
        finally:
            self._host_io = None
        if self._last_stepwise:  # redone stage by stage: copy its force out
            b.copy_(self.b)
        return res

    def _capture(self, key):
        if key[-1]:  # periodic rebuilds alternate with refits: not one fixed sequence
            return
        g = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with N.no_collection(), torch.cuda.graph(g):
            self._enqueue()
        self._graph = (key, g)

    def _enqueue(self):
        """All stages of iteration(), ending with the copies of counts,
        status, energy and TOI into pinned host memory, on four streams: the
        triangle side (box refit, PT query, PT records) beside the edge side,
        and each CCD query (swept boxes, refit, TOI; own candidate workspace)
        as soon as the discrete query on its hierarchy is done, beside the
        narrow phase, the contact BSR and the energy.  Nothing after the
        discrete queries reads the hierarchies, so the CCD refits cannot
        disturb them; every stream joins the first before the read."""
        if getattr(self, "bvh_rebuild_interval", 0) or not self.has_triangles:
            return self._enqueue_serial()
        ee, pt = self.contacts_new, self.contacts_pt
        main = torch.cuda.current_stream()
        side, ccd_e, ccd_t = self._side, self._ccd_e, self._ccd_t
        soup = ctypes.byref(self.soup.c_struct())
        kappa = float(self.contact_stiffness)
        excl = int(self.disable_self_collision)
        pad = 1e-7
        cap = ee.capacity + pt.capacity
        t = self.collision_triplets
        if t is None or t.rows.shape[0] < 16 * cap:
            t = self.collision_triplets = Triplets.zeros(16 * cap, self.soup.xcs.dtype, self.device)
        self._ws_ee = hessian_workspace(ee, getattr(self, "_ws_ee", None))
        self._ws_pt = hessian_workspace(pt, getattr(self, "_ws_pt", None))
        io = self._host_io
        if io is not None:
            self.soup.x_transformed.copy_(io[0], non_blocking=True)
        self.compute_V(ret=False)
        self._pack()
        self.b.zero_()
        self.ccd_toi.fill_(1.0)
        self._status.zero_()
        if io is None:
            N.call("ipcb_add_dx", soup, N.ptr(self._dx_buf), N.ptr(self.ccd_x1), N.stream_handle())
        else:  # the direction crosses the bus beside the discrete queries
            cin = self._copy_in
            cin.wait_stream(main)
            with torch.cuda.stream(cin):
                self._dx_buf.copy_(io[1], non_blocking=True)
                N.call("ipcb_add_dx", soup, N.ptr(self._dx_buf), N.ptr(self.ccd_x1), N.stream_handle())
                self._x1_done.record(cin)
        side.wait_stream(main)
        with torch.cuda.stream(side):
            self._triangle_aabbs()
            self.tri_mesh.refit()
            self._launch_dcd("pt")
            self._pt_done.record(side)
        N.call("ipcb_edge_aabbs", soup, N.ptr(self.x4), float(contact._thickness + contact.buffer),
               N.ptr(self.bvh_edges_lower), N.ptr(self.bvh_edges_upper), N.stream_handle())
        self.bvh_edges.refit()
        self._launch_dcd("ee")
        self._ee_done.record(main)
        with torch.cuda.stream(ccd_e):
            ccd_e.wait_event(self._ee_done)
            if io is not None:
                ccd_e.wait_event(self._x1_done)
            s1 = N.stream_handle()
            N.call("ipcb_swept_edge_aabbs", soup, N.ptr(self.ccd_x1), pad, N.ptr(self.ccd_edge_lower),
                   N.ptr(self.ccd_edge_upper), s1)
            self.ccd_edge_bvh.refit(self.ccd_edge_lower, self.ccd_edge_upper)
            N.call("ipcb_edge_edge_toi", soup, N.ptr(self.ccd_x1), ctypes.byref(self.ccd_edge_bvh.c),
                   N.ptr(self.ccd_edge_lower), N.ptr(self.ccd_edge_upper), excl, N.ptr(self.ccd_toi),
                   N.ptr(self._status), N.ptr(self._toi_ws), self._toi_ws.numel(), s1)
        with torch.cuda.stream(ccd_t):
            ccd_t.wait_event(self._pt_done)
            if io is not None:
                ccd_t.wait_event(self._x1_done)
            s2 = N.stream_handle()
            N.call("ipcb_swept_triangle_aabbs", soup, N.ptr(self.ccd_x1), pad, N.ptr(self.ccd_triangle_lower),
                   N.ptr(self.ccd_triangle_upper), s2)
            self.ccd_triangle_bvh.refit(self.ccd_triangle_lower, self.ccd_triangle_upper)
            N.call("ipcb_point_triangle_toi", soup, N.ptr(self.ccd_x1), ctypes.byref(self.ccd_triangle_bvh.c), pad,
                   excl, N.ptr(self.ccd_toi), N.ptr(self._status), N.ptr(self._toi_ws_pt),
                   self._toi_ws_pt.numel(), s2)
        contact_hessian_ee(self.states, self.soup, ee, t, self.b, kappa, n=-1, ws=self._ws_ee)
        with torch.cuda.stream(side):
            side.wait_event(self._ee_done)  # the PT records follow the EE count
            contact_hessian_pt_after(self.states, self.soup, pt, t, self.b, ee, kappa, ws=self._ws_pt)
        main.wait_stream(side)
        if io is not None:  # the force is final: send it back beside the remaining stages
            cout = self._copy_out
            cout.wait_stream(main)
            with torch.cuda.stream(cout):
                io[2].copy_(self.b, non_blocking=True)
        H, _ = contact_bsr(ee, None, pt, None, self.soup.n_verts, t, out=self.collision_hessian,
                           status=self._bsr_status, read_status=False)
        self.collision_hessian = H
        e = self._energy.zero_()
        contact_energy_ee(self.states, self.soup, ee, e, kappa, n=-1)
        contact_energy_pt(self.states, self.soup, pt, e, kappa, n=-1)
        main.wait_stream(ccd_e)
        main.wait_stream(ccd_t)
        if io is not None:
            main.wait_stream(self._copy_in)
            main.wait_stream(self._copy_out)
        self._copy_results(e)

    def _copy_results(self, e):
        ee, pt = self.contacts_new, self.contacts_pt
        h = self._readback
        h["counts"][0:1].copy_(ee.cnt, non_blocking=True)
        h["counts"][1:2].copy_(pt.cnt, non_blocking=True)
        h["counts"][2:3].copy_(self._bsr_status, non_blocking=True)
        h["counts"][3:4].copy_(self._status, non_blocking=True)
        h["energy"].copy_(e, non_blocking=True)
        h["toi"].copy_(self.ccd_toi, non_blocking=True)

    def _enqueue_serial(self):
        """_enqueue on one stream (periodic BVH rebuilds, or no triangles)."""
        ee, pt = self.contacts_new, self.contacts_pt
        io = self._host_io
        if io is not None:
            self.soup.x_transformed.copy_(io[0], non_blocking=True)
            self._dx_buf.copy_(io[1], non_blocking=True)
        self.compute_V(ret=False)
        self._status.zero_()
        self.update_bvh()
        self._launch_dcd("ee")
        if self.has_triangles:
            self._launch_dcd("pt")
        else:
            pt.cnt.zero_()
        cap = ee.capacity + pt.capacity
        t = self.collision_triplets
        if t is None or t.rows.shape[0] < 16 * cap:
            t = self.collision_triplets = Triplets.zeros(16 * cap, self.soup.xcs.dtype, self.device)
        kappa = float(self.contact_stiffness)
        self.b.zero_()
        self._ws_ee = hessian_workspace(ee, getattr(self, "_ws_ee", None))
        self._ws_pt = hessian_workspace(pt, getattr(self, "_ws_pt", None))
        contact_hessian_ee(self.states, self.soup, ee, t, self.b, kappa, n=-1, ws=self._ws_ee)
        contact_hessian_pt_after(self.states, self.soup, pt, t, self.b, ee, kappa, ws=self._ws_pt)
        H, _ = contact_bsr(ee, None, pt, None, self.soup.n_verts, t, out=self.collision_hessian,
                           status=self._bsr_status, read_status=False)
        self.collision_hessian = H
        e = self._energy.zero_()
        contact_energy_ee(self.states, self.soup, ee, e, kappa, n=-1)
        contact_energy_pt(self.states, self.soup, pt, e, kappa, n=-1)
        self._launch_ccd(self._dx_buf, reset_status=False)
        if io is not None:
            io[2].copy_(self.b, non_blocking=True)
        self._copy_results(e)

    def iteration_stepwise(self) -> IterationResult:
        """The same iteration through the public calls, one stage at a time
        (each reads its counts or result on the host)."""
        self.detect_collision()
        self.b.zero_()
        self.compute_contact_hessian(detect=False)
        e = self.compute_collision_energy(detect=False)
        dcd_status = self.query_status
        alpha = self.line_search_upper_bound()
        return IterationResult(self.n_contacts, self.n_contacts_pt, e, alpha, dcd_status | self.query_status)

    def set_positions(self, x) -> None:
        if isinstance(x, np.ndarray):
            x = torch.from_numpy(x)
        self.soup.x_transformed.copy_(x, non_blocking=True)
