"""One scene's per-Newton-iteration contact work split over several GPUs, one
process per GPU (the reference is single-GPU; this is how its contact
pipeline shards).

Positions, the hierarchies and the surface are replicated: every rank refits
its own copy.  The queries are split by index: the edge-edge queries (DCD and
CCD) by Morton rank in the edge hierarchy -- every pair is met by its
lower-ranked edge, so disjoint rank ranges partition the pair set -- and the
point-triangle queries by vertex.  Each rank runs the narrow phase on its own
records (its share of the 16-block triplets and of the contact BSR: the
matrix is the sum of the ranks' matrices) and the exchange is one step:

* the vertex force (the gradient's contact part): all-reduce, sum;
* the barrier energy: all-reduce, sum;
* the CCD time of impact: all-reduce, minimum; the query status words: OR;
* the record counts: all-reduce, sum (the global pair count).

``shard_range`` is the partition, ``combine`` the exchange (both testable
without a GPU), ``ShardedContactPipeline.iteration`` the per-rank sequence.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import _native as N
from . import contact
from .bsr import Triplets, contact_bsr
from .contact import QUERY_FAILED, Soup
from .dynamic_contacts import (ContactBarrierMixin, contact_energy_ee, contact_energy_pt, contact_hessian_ee,
                               contact_hessian_pt, hessian_workspace)


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """(first, count) of rank's contiguous share of n queries; the shares
    differ in size by at most one and cover 0 .. n - 1 once."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard {rank} of {world} over {n}")
    base, rem = divmod(n, world)
    return rank * base + min(rank, rem), base + (1 if rank < rem else 0)


@dataclass
class ShardResult:
    n_ee: int          # this rank's records
    n_pt: int
    n_ee_total: int    # all ranks' records
    n_pt_total: int
    energy: float      # barrier energy of the scene (all ranks), times h^2
    alpha: float       # the scene's CCD step bound
    status: int        # OR of every rank's query status bits


def combine(force: torch.Tensor, scalars: torch.Tensor, toi: torch.Tensor, status: torch.Tensor, group=None):
    """The exchange step, in place: force (V, 3) and scalars (energy, n_ee,
    n_pt as float64) summed over the ranks, toi (1,) their minimum, status
    (1,) int32 the OR of theirs.  Works on any backend the tensors' device
    supports (NCCL for CUDA tensors, gloo for CPU tensors)."""
    import torch.distributed as dist

    dist.all_reduce(force, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(scalars, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(toi, op=dist.ReduceOp.MIN, group=group)
    world = dist.get_world_size(group)
    words = [torch.zeros_like(status) for _ in range(world)]
    dist.all_gather(words, status, group=group)
    acc = torch.zeros_like(status)
    for w in words:
        acc = acc | w
    status.copy_(acc)


class ShardedContactPipeline(ContactBarrierMixin):
    """ContactPipeline.iteration for rank ``rank`` of ``world``.  With
    ``exchange=False`` the collectives are skipped and the result is the
    rank's own share (the single-process check of the partition uses it)."""

    def __init__(self, soup: Soup, dhat: float, kappa: float, rank: int, world: int, h: float = 1e-2,
                 exclude_same_body: bool = False, group=None, exchange: bool = True):
        contact._thickness = 0.5 * dhat
        contact.buffer = 0.5 * dhat
        self.soup = soup
        self.h = float(h)
        self.contact_stiffness = float(kappa)
        self.rank, self.world, self.group, self.exchange = int(rank), int(world), group, bool(exchange)
        self.b = torch.zeros_like(soup.x_transformed)
        ContactBarrierMixin.__init__(self)
        self.disable_self_collision = exclude_same_body
        self.ee_range = shard_range(soup.n_edges, self.rank, self.world)
        self.pt_range = shard_range(soup.n_verts, self.rank, self.world)
        self.collision_triplets = None
        self.collision_hessian = None
        dev = soup.x_transformed.device
        self._scalars = torch.zeros(3, dtype=torch.float64, device=dev)
        self._energy = torch.zeros(1, dtype=torch.float64, device=dev)

    @classmethod
    def from_scene(cls, scene, rank: int, world: int, dtype=None, device="cuda", **kw) -> "ShardedContactPipeline":
        soup = Soup.from_numpy(scene.x, scene.edges, scene.triangles, scene.body, xcs=scene.xcs, device=device,
                               dtype=dtype)
        return cls(soup, scene.dhat, scene.kappa, rank, world, **kw)

    # ---------------------------------------------------- ranged queries
    def _launch_dcd(self, which: str):
        soup = self.soup.c_struct()
        s = N.stream_handle()
        th = float(contact._thickness)
        if which == "ee":
            self.contacts_new.cnt.zero_()
            first, count = self.ee_range
            N.call("ipcb_dcd_ee_range", ctypes.byref(soup), N.ptr(self.x4), ctypes.byref(self.bvh_edges.c), th,
                   float(contact._thickness + contact.buffer), int(self.disable_self_collision), first, count,
                   ctypes.byref(self.contacts_new.c_struct()), N.ptr(self._status), s)
        else:
            self.contacts_pt.cnt.zero_()
            first, count = self.pt_range
            N.call("ipcb_dcd_pt_range", ctypes.byref(soup), N.ptr(self.x4), ctypes.byref(self.tri_mesh.c), th,
                   float(2.0 * (contact._thickness + contact.buffer)), int(self.disable_self_collision), None, first,
                   count, ctypes.byref(self.contacts_pt.c_struct()), N.ptr(self._status), s)

    def _launch_ccd(self, dx: torch.Tensor, reset_status: bool = True):
        soup = self.soup.c_struct()
        s = N.stream_handle()
        pad = 1e-7
        excl = int(self.disable_self_collision)
        N.call("ipcb_add_dx", ctypes.byref(soup), N.ptr(dx), N.ptr(self.ccd_x1), s)
        self.ccd_toi.fill_(1.0)
        if reset_status:
            self._status.zero_()
        N.call("ipcb_swept_edge_aabbs", ctypes.byref(soup), N.ptr(self.ccd_x1), pad, N.ptr(self.ccd_edge_lower),
               N.ptr(self.ccd_edge_upper), s)
        self.ccd_edge_bvh.refit(self.ccd_edge_lower, self.ccd_edge_upper)
        first, count = self.ee_range
        N.call("ipcb_edge_edge_toi_range", ctypes.byref(soup), N.ptr(self.ccd_x1), ctypes.byref(self.ccd_edge_bvh.c),
               N.ptr(self.ccd_edge_lower), N.ptr(self.ccd_edge_upper), excl, first, count, N.ptr(self.ccd_toi),
               N.ptr(self._status), N.ptr(self._toi_ws), self._toi_ws.numel(), s)
        if self.has_triangles:
            N.call("ipcb_swept_triangle_aabbs", ctypes.byref(soup), N.ptr(self.ccd_x1), pad,
                   N.ptr(self.ccd_triangle_lower), N.ptr(self.ccd_triangle_upper), s)
            self.ccd_triangle_bvh.refit(self.ccd_triangle_lower, self.ccd_triangle_upper)
            first, count = self.pt_range
            N.call("ipcb_point_triangle_toi_range", ctypes.byref(soup), N.ptr(self.ccd_x1),
                   ctypes.byref(self.ccd_triangle_bvh.c), pad, excl, first, count, N.ptr(self.ccd_toi),
                   N.ptr(self._status), N.ptr(self._toi_ws), self._toi_ws.numel(), s)

    # --------------------------------------------------------- iteration
    def iteration(self, dx: torch.Tensor) -> ShardResult:
        """This rank's share of one Newton iteration's contact work, then the
        exchange: detect (ranged), 16 triplets per local record and the local
        force, the local contact BSR, the barrier energy, the ranged CCD."""
        self.detect_collision()
        dcd_status = self.query_status
        n_ee, n_pt = self.n_contacts, self.n_contacts_pt
        nc = 16 * (n_ee + n_pt)
        t = self.collision_triplets
        if t is None or t.rows.shape[0] < nc:
            t = self.collision_triplets = Triplets.zeros(max(nc, 16), self.soup.xcs.dtype, self.device)
        kappa = float(self.contact_stiffness)
        self.b.zero_()
        if n_ee:
            self._ws_ee = hessian_workspace(self.contacts_new, getattr(self, "_ws_ee", None))
            contact_hessian_ee(None, self.soup, self.contacts_new, t, self.b, kappa, n=n_ee, ws=self._ws_ee)
        if n_pt:
            self._ws_pt = hessian_workspace(self.contacts_pt, getattr(self, "_ws_pt", None))
            contact_hessian_pt(None, self.soup, self.contacts_pt, t, self.b, n_ee, kappa, n=n_pt, ws=self._ws_pt)
        H, _ = contact_bsr(self.contacts_new, n_ee, self.contacts_pt, n_pt, self.soup.n_verts, t,
                           out=self.collision_hessian, read_status=False)
        self.collision_hessian = H
        e = self._energy.zero_()
        if n_ee:
            contact_energy_ee(None, self.soup, self.contacts_new, e, kappa, n=n_ee)
        if n_pt:
            contact_energy_pt(None, self.soup, self.contacts_pt, e, kappa, n=n_pt)
        self._launch_ccd(dx, reset_status=False)
        sc = self._scalars
        sc[0:1].copy_(e)
        sc[1] = float(n_ee)
        sc[2] = float(n_pt)
        toi = self.ccd_toi.double()
        status = self._status.clone()
        if self.exchange and self.world > 1:
            combine(self.b, sc, toi, status, self.group)
        vals = torch.cat([sc, toi, status.double()]).tolist()
        energy, ee_tot, pt_tot, toi_v, st = vals[0], int(vals[1]), int(vals[2]), vals[3], int(vals[4])
        st |= dcd_status
        self.query_status = st
        alpha = 0.0 if st & QUERY_FAILED else (0.9 * toi_v if toi_v < 1.0 else 1.0)
        return ShardResult(n_ee, n_pt, ee_tot, pt_tot, energy * self.h * self.h, alpha, st)
