"""Implicit-Euler Newton integrator with IPC contact: the time integrator of
time_integrator_base.py:375-546 (``RodBCBase.step``, ``compute_A``,
``compute_rhs``, ``solve``, ``line_search``) and the contact parts of
``RodComplexBC`` (dynamic_contacts.py:249-308), on the GPU kernels of this
package.

Per Newton iteration:
  A  = M + h^2 (K + C) + h^2 k_att I_fixed          (BSR, one assembly)
  b  = -h^2 (f_elastic + f_contact) + M (x - x~) + h^2 k_att (x - x_target)_fixed
  A dx = b  by PCG (relative residual ``tol``, ``maxiter``; block-Jacobi or a
            learned preconditioner), direct solve when PCG misses the tolerance
  x -= alpha dx, alpha from the CCD bound and backtracking on the total energy
  E = h^2 Psi + 1/2 |x - x~|_M^2 + h^2 B_contact + 1/2 h^2 k_att |x - x_target|^2
(energies and the convergence norm max|dx| in double).  x~ = x0 + h xdot + h^2 g.
"""
from __future__ import annotations

import ctypes
import gc
import math
import warnings
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from . import contact as contact_mod
from .autotune import Autotuner, bucket
from .bsr import BsrMatrix, Triplets, bsr_from_triplets, bsr_mv, contact_bsr
from .contact import QUERY_FAILED, Soup
from .dynamic_contacts import (ContactBarrierMixin, contact_hessian_ee, contact_hessian_pt, contact_hessian_pt_after,
                               hessian_workspace)

MATERIALS = {"snh": 0, "neo_hookean": 1, "nh": 1, "stvk": 2}


def lame(E: float, nu: float):
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


@dataclass
class NewtonState:
    """fem/params.py:43-50."""
    x: torch.Tensor
    x0: torch.Tensor
    dx: torch.Tensor
    xdot: torch.Tensor


@dataclass
class StepStats:
    newton_iterations: int = 0
    pcg_iterations: list = field(default_factory=list)
    fallbacks: int = 0
    direct_failures: int = 0
    alphas: list = field(default_factory=list)
    energies: list = field(default_factory=list)
    norms: list = field(default_factory=list)
    ccd_refusals: int = 0  # line searches refused because a CCD query ran out of its bounds


class BlockJacobi:
    """Inverse of the 3x3 diagonal blocks of a BSR matrix."""

    def __init__(self, A: BsrMatrix):
        nnz = A.nnz_sync()
        rows = torch.repeat_interleave(torch.arange(A.nrow, device=A.device),
                                       (A.offsets[1:] - A.offsets[:-1]).long())
        diag = rows == A.columns[:nnz].long()
        D = torch.zeros((A.nrow, 3, 3), dtype=torch.float64, device=A.device)
        D[rows[diag]] = A.values[:nnz][diag].double()
        eye = torch.eye(3, dtype=torch.float64, device=A.device)
        D = torch.where(D.abs().sum(dim=(1, 2), keepdim=True) > 0, D, eye)
        self.Dinv = torch.linalg.inv(D).to(A.dtype)

    def __call__(self, r: torch.Tensor) -> torch.Tensor:
        return torch.bmm(self.Dinv, r.unsqueeze(-1)).squeeze(-1)


def pcg(A: BsrMatrix, b: torch.Tensor, precond, tol: float = 1e-6, maxiter: int = 200):
    """Preconditioned CG on the (V, 3) block vector b; dot products in double.
    Returns (x, iterations, relative residual)."""
    x = torch.zeros_like(b)
    r = b.clone()
    bn = float(torch.linalg.vector_norm(b.double()))
    if bn == 0.0:
        return x, 0, 0.0
    z = precond(r)
    p = z.clone()
    rz = float((r.double() * z.double()).sum())
    Ap = torch.empty_like(b)
    rel = 1.0
    for it in range(1, maxiter + 1):
        bsr_mv(A, p, Ap)
        pAp = float((p.double() * Ap.double()).sum())
        if not (pAp > 0.0):
            return x, it, float("nan")
        a = rz / pAp
        x.add_(p, alpha=a)
        r.sub_(Ap, alpha=a)
        rel = float(torch.linalg.vector_norm(r.double())) / bn
        if rel <= tol:
            return x, it, rel
        z = precond(r)
        rz_new = float((r.double() * z.double()).sum())
        p.mul_(rz_new / rz).add_(z)
        rz = rz_new
    return x, maxiter, rel


class JacobiPrecond:
    """Block-Jacobi preconditioner for DevicePcg (inverse diagonal blocks);
    ``out`` reuses a buffer, so that a graph-replayed PCG keeps its pointers.

    ``groups=(n_point, n_groups)``: block rows n_point + 4 g .. + 3 form one
    group (an affine body's p, a0, a1, a2) preconditioned by the inverse of
    their 12x12 diagonal block (ipcb_group_jacobi); ``out_group`` reuses that
    buffer."""
    kind = 0

    def __init__(self, A: BsrMatrix, out: torch.Tensor | None = None, groups: tuple[int, int] | None = None,
                 out_group: torch.Tensor | None = None):
        shape = (A.nrow, 3, 3)
        ok = out is not None and tuple(out.shape) == shape and out.dtype == A.dtype
        self.dinv = out if ok else torch.empty(shape, dtype=A.dtype, device=A.device)
        status = torch.zeros(1, dtype=torch.int32, device=A.device)
        fp64 = int(A.dtype == torch.float64)
        N.call("ipcb_block_jacobi", A.nrow, N.ptr(A.offsets), N.ptr(A.columns), None, N.ptr(A.values), fp64,
               N.ptr(self.dinv), N.ptr(status), N.stream_handle())
        self.n_point, self.n_groups = groups if groups else (A.nrow, 0)
        self.dinv_group = None
        if self.n_groups:
            if self.n_point + 4 * self.n_groups != A.nrow:
                raise ValueError(f"groups {groups} do not cover {A.nrow} block rows")
            gshape = (self.n_groups, 12, 12)
            ok = out_group is not None and tuple(out_group.shape) == gshape and out_group.dtype == A.dtype
            self.dinv_group = out_group if ok else torch.empty(gshape, dtype=A.dtype, device=A.device)
            N.call("ipcb_group_jacobi", self.n_point, self.n_groups, N.ptr(A.offsets), N.ptr(A.columns),
                   N.ptr(A.values), fp64, N.ptr(self.dinv_group), N.ptr(status), N.stream_handle())

    def fill(self, P):
        P.dinv = N.ptr(self.dinv)
        P.n_point, P.n_groups = self.n_point, self.n_groups
        P.dinv_group = N.ptr(self.dinv_group) if self.n_groups else None


class DevicePcg:
    """PCG with device-resident scalars (ipcb_pcg_*): ``batch`` iterations
    per host check, replayed from a CUDA graph captured once per set of
    buffers; one synchronisation per batch."""

    def __init__(self, batch: int = 16, use_graph: bool = True):
        self.batch = batch
        self.use_graph = use_graph
        self._bufs = None
        self._graph = None
        self._key = None

    def _buffers(self, n, dtype, device):
        if self._bufs is None or self._bufs["n"] != n or self._bufs["dtype"] != dtype:
            z = lambda: torch.zeros((n, 3), dtype=dtype, device=device)
            self._bufs = dict(n=n, dtype=dtype, x=z(), r=z(), z=z(), p=z(), q=z(), t=z(), b=z(), x0=z(),
                              state=torch.zeros(ctypes.sizeof(N.PcgState), dtype=torch.uint8, device=device),
                              host=torch.zeros(ctypes.sizeof(N.PcgState), dtype=torch.uint8).pin_memory())
        return self._bufs

    def solve(self, A: BsrMatrix, b: torch.Tensor, M, tol: float, maxiter: int, x0: torch.Tensor | None = None):
        """Returns (x, iterations, relative residual, status); x is a view of
        an internal buffer (valid until the next solve).  x0: initial guess
        (None: zero); the stopping test stays relative to |b|."""
        n = A.nrow
        B = self._buffers(n, A.dtype, A.device)
        B["b"].copy_(b)
        P = N.Pcg()
        P.n, P.fp64, P.precond = n, int(A.dtype == torch.float64), M.kind
        P.offsets, P.columns, P.values = N.ptr(A.offsets), N.ptr(A.columns), N.ptr(A.values)
        for k in ("b", "x", "r", "z", "p", "q", "t"):
            setattr(P, k, N.ptr(B[k]))
        P.state = N.ptr(B["state"])
        M.fill(P)
        if x0 is not None:
            B["x0"].copy_(x0.reshape(n, 3))
            P.x0 = N.ptr(B["x0"])
        self._P = P
        N.call("ipcb_pcg_start", ctypes.byref(P), float(tol), int(maxiter), N.stream_handle())
        key = tuple(getattr(P, f) for f, _ in N.Pcg._fields_ if f != "x0")  # the loop never reads x0
        if self.use_graph and key != self._key:
            self._graph = torch.cuda.CUDAGraph()
            with N.no_collection(), torch.cuda.graph(self._graph):
                N.call("ipcb_pcg_iterate", ctypes.byref(P), self.batch, N.stream_handle())
            self._key = key
        st = N.PcgState()
        while True:
            if self.use_graph:
                self._graph.replay()
            else:
                N.call("ipcb_pcg_iterate", ctypes.byref(P), self.batch, N.stream_handle())
            B["host"].copy_(B["state"], non_blocking=True)
            torch.cuda.current_stream().synchronize()
            st = N.PcgState.from_buffer_copy(B["host"].numpy().tobytes())
            if st.done:
                break
        if x0 is not None and not st.bb > 0:
            B["x"].zero_()  # b = 0: the solution is 0, whatever the guess
        rel = math.sqrt(st.last_rr / st.bb) if st.bb > 0 else 0.0
        return B["x"], st.it, rel, st.status


def terms_candidates() -> list[tuple]:
    """Schedules of the per-iteration terms: the per-kind kernels back to
    back ("separate"), or the one persistent work-queue launch
    (ipcb_terms_launch) as (register variant, blocks per SM, threads, tile)."""
    shapes = [(0, bps, 128) for bps in (1, 2, 3)] + [(1, bps, 128) for bps in (1, 2)] + \
        [(v, 4, 64) for v in (0, 1)]
    return [("separate",)] + [(v, bps, th, tile) for (v, bps, th) in shapes for tile in (32, 64, 128)]


def launch_terms(Tc, cfg, n_sm: int):
    variant, bps, threads, tile = cfg
    N.call("ipcb_terms_launch", ctypes.byref(Tc), bps * n_sm, threads, tile, variant, N.stream_handle())


class FEMContactSolver(ContactBarrierMixin):
    """Deformable bodies (tet FEM) with IPC contact: RodComplexBC on the GPU."""

    def __init__(self, scene, *, material: str = "neo_hookean", E: float = 1e5, nu: float = 0.4, rho: float = 1000.0,
                 gravity=(0.0, -9.8, 0.0), h: float = 1e-2, fixed: np.ndarray | None = None,
                 attachment_stiffness: float = 1e11, dtype=torch.float32, device="cuda", vel_tol: float = 5e-2,
                 max_newton: int = 100, tol: float = 1e-4, maxiter: int = 200, exclude_same_body: bool = False,
                 linear_solver: str = "pcg", direct_fallback: bool = True, preconditioner: str = "jacobi",
                 precond_refresh: int = 1, assembly: str = "queue", line_search_mode: str = "device"):
        self.h = float(h)
        if line_search_mode not in ("device", "host"):
            raise ValueError(f"unknown line search mode {line_search_mode!r}")
        # "device": trials in one CUDA graph WHILE loop, one read per search
        # (csrc/linesearch.cu); "host": the reference's loop with host reads
        self.line_search_mode = line_search_mode
        self._ls = None
        if assembly not in ("queue", "generic"):
            raise ValueError(f"unknown assembly {assembly!r}")
        # "queue": one persistent launch for contact + tet terms and the
        # fixed-pattern assembly (csrc/terms.cu); "generic": per-term kernels
        # and a sort-based assembly of all triplets
        self.assembly = assembly
        # queue assembly: replay compute_A from a CUDA graph (device-side
        # counts, one host read) once a step-by-step call has sized the buffers
        self.graph_compute_A = True
        self._static = None
        self.material = MATERIALS[material]
        self.mu, self.lam = lame(E, nu)
        self.dtype = dtype
        self.device = torch.device(device)
        self.vel_tol, self.max_newton = vel_tol, max_newton
        self.tol, self.maxiter = tol, maxiter
        self.contact_stiffness = float(scene.kappa)
        contact_mod._thickness = 0.5 * scene.dhat
        contact_mod.buffer = 0.5 * scene.dhat
        self.soup = Soup.from_numpy(scene.x, scene.edges, scene.triangles, scene.body, xcs=scene.xcs,
                                    device=self.device, dtype=dtype)
        V = self.soup.n_verts
        self.tets = torch.as_tensor(scene.tets, dtype=torch.int32, device=self.device).contiguous()
        self.n_tets = self.tets.shape[0]
        self.Bm = torch.zeros((self.n_tets, 3, 3), dtype=dtype, device=self.device)
        self.W = torch.zeros(self.n_tets, dtype=dtype, device=self.device)
        fp64 = int(dtype == torch.float64)
        N.call("ipcb_tet_rest", fp64, N.ptr(self.soup.xcs), N.ptr(self.tets), self.n_tets, N.ptr(self.Bm), N.ptr(self.W),
               N.stream_handle())
        # lumped mass: rho * volume / 4 per tet vertex
        w = self.W.double().cpu().numpy()
        m = np.zeros(V)
        np.add.at(m, scene.tets.reshape(-1), np.repeat(rho * w / 4.0, 4))
        m[m == 0] = rho * (w.mean() if len(w) else 1.0) / 4.0
        self.mass = torch.tensor(m, dtype=torch.float64, device=self.device)
        self.gravity = torch.tensor(gravity, dtype=torch.float64, device=self.device)
        x = self.soup.x_transformed
        self.states = NewtonState(x=x, x0=x.clone(), dx=torch.zeros_like(x), xdot=torch.zeros_like(x))
        self.b = torch.zeros_like(x)
        self.fixed = torch.zeros(V, dtype=torch.bool, device=self.device)
        if fixed is not None:
            self.fixed = torch.as_tensor(fixed, dtype=torch.bool, device=self.device)
        self.x_target = self.soup.xcs.clone()
        self.k_att = float(attachment_stiffness)
        ContactBarrierMixin.__init__(self)
        self.disable_self_collision = exclude_same_body
        self._elastic = Triplets.zeros(16 * self.n_tets, dtype, self.device)
        # precond_factory: host-loop preconditioner (``pcg``); device_precond:
        # the same preconditioner for DevicePcg
        if preconditioner == "jacobi":
            self.precond_factory = BlockJacobi
            self._dinv = None

            def jacobi(A):
                p = JacobiPrecond(A, self._dinv)
                self._dinv = p.dinv
                return p

            self.device_precond = jacobi
        elif preconditioner == "learned":
            from .learned import DEFAULT_WEIGHTS, LearnedFactor, LearnedPreconditioner, Net

            net = Net.load(DEFAULT_WEIGHTS, device=self.device)
            self.precond_factory = LearnedPreconditioner(net)
            from .learned import Pool

            self._factor_pool = Pool()
            self.device_precond = lambda A: LearnedFactor(net, A, pool=self._factor_pool)
        else:
            raise ValueError(f"unknown preconditioner {preconditioner!r}")
        self.host_pcg = False
        self.device_pcg = DevicePcg()
        # the learned factor is rebuilt every `precond_refresh` Newton
        # iterations (and at the first iteration of a step); in between the
        # previous factor preconditions the new matrix
        self.precond_refresh = max(int(precond_refresh), 1)
        self._precond = None
        self._precond_age = 0
        if linear_solver not in ("pcg", "direct"):
            raise ValueError(f"unknown linear solver {linear_solver!r}")
        self.linear_solver = linear_solver
        self.direct_fallback = direct_fallback
        self.direct_solver = None  # DirectSolver, created on first use
        self.frame = 0
        self.time = 0.0
        # prescribed boundary (compute_compensation, time_integrator_base.py:440-467):
        # callable(t) -> (V, 3) attachment targets of the fixed vertices at time t
        self.boundary = None
        self.stats = StepStats()

    # ----------------------------------------------------------- energies
    def x_tilde(self) -> torch.Tensor:
        h = self.h
        return self.states.x0.double() + h * self.states.xdot.double() + h * h * self.gravity

    def elastic_energy(self) -> float:
        e = torch.zeros(1, dtype=torch.float64, device=self.device)
        N.call("ipcb_tet_energy", self.material, int(self.dtype == torch.float64), N.ptr(self.states.x),
               N.ptr(self.tets), self.n_tets, N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, N.ptr(e),
               N.stream_handle())
        return float(e.item())

    def total_energy(self) -> float:
        """h^2 Psi + inertia + h^2 contact + attachment, in double (line search)."""
        h2 = self.h * self.h
        x = self.states.x.double()
        d = x - self.x_tilde()
        inertia = 0.5 * float((self.mass[:, None] * d * d).sum())
        att = 0.0
        if bool(self.fixed.any()):
            r = (x - self.x_target.double())[self.fixed]
            att = 0.5 * self.k_att * h2 * float((r * r).sum())
        return h2 * self.elastic_energy() + inertia + self.compute_collision_energy() + att

    # ------------------------------------------------------------ system
    def compute_A(self) -> BsrMatrix:
        """time_integrator_base.py:406-426 + dynamic_contacts.py:275-297."""
        if self.assembly == "queue":
            if self.graph_compute_A and self.device.type == "cuda" and not getattr(self, "bvh_rebuild_interval", 0):
                return self._compute_A_graph()
            return self._compute_A_queue()
        return self._compute_A_generic()

    # ------------------------------------------ graph-replayed compute_A
    def _graph_buffers(self):
        """Buffers sized for the list capacities (so the captured launches
        never need a count on the host): the contact triplets, the contact
        BSR and the union (static pattern + 16 blocks per possible record)."""
        st = self._static
        ee, pt = self.contacts_new, self.contacts_pt
        cap_rec = ee.capacity + pt.capacity
        t = self.collision_triplets
        if t is None or t.rows.shape[0] < 16 * cap_rec:
            self.collision_triplets = Triplets.zeros(16 * cap_rec, self.dtype, self.device)
        V = self.soup.n_verts
        cap = st["nnz"] + 16 * cap_rec
        A = getattr(self, "A", None)
        if A is None or A.columns.shape[0] < cap or "a_rows" not in st or st["a_rows"].shape[0] < cap:
            A = self.A = BsrMatrix(V, V, cap, self.dtype, self.device)
            for k in ("a_rows", "src_a", "src_b"):
                st[k] = torch.empty(cap, dtype=torch.int32, device=self.device)
        if "graph_read" not in st:
            st["graph_read"] = torch.zeros(4, dtype=torch.int32, pin_memory=True)
        return min(A.columns.shape[0], st["a_rows"].shape[0])

    def _enqueue_A(self, cfg, cap: int):
        """compute_A's launches with every count read on the device: box
        refits and the discrete queries, the per-iteration terms on schedule
        ``cfg``, the contact BSR of the lists' capacities, the union with the
        elastic pattern and its values; ends with the copy of the two list
        counts and the two status words into pinned host memory."""
        st = self._static
        h2 = self.h * self.h
        V = self.soup.n_verts
        ee, pt = self.contacts_new, self.contacts_pt
        t = self.collision_triplets
        s = N.stream_handle()
        self.b.zero_()
        self.compute_V(ret=False)
        self._status.zero_()
        self.update_bvh()
        self._launch_dcd("ee")
        if self.has_triangles:
            self._launch_dcd("pt")
        else:
            pt.cnt.zero_()
        kappa = float(self.contact_stiffness)
        if cfg[0] == "separate":
            self._ws_ee = hessian_workspace(ee, getattr(self, "_ws_ee", None))
            self._ws_pt = hessian_workspace(pt, getattr(self, "_ws_pt", None))
            contact_hessian_ee(None, self.soup, ee, t, self.b, kappa, n=-1, ws=self._ws_ee)
            contact_hessian_pt_after(None, self.soup, pt, t, self.b, ee, kappa, ws=self._ws_pt)
            N.call("ipcb_tet_hessian", self.material, int(self.dtype == torch.float64), N.ptr(self.states.x),
                   N.ptr(self.tets), self.n_tets, N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, None, None,
                   N.ptr(st["tet_vals"]), N.ptr(self.b), s)
        else:
            Tc = N.Terms(int(self.dtype == torch.float64), N.ptr(self.states.x), N.ptr(self.soup.xcs),
                         ee.c_struct(), pt.c_struct(), kappa, N.ptr(t.rows), N.ptr(t.cols), N.ptr(t.vals),
                         N.ptr(t.mask), self.material, N.ptr(self.tets), self.n_tets, N.ptr(self.Bm), N.ptr(self.W),
                         self.mu, self.lam, None, None, N.ptr(st["tet_vals"]), N.ptr(self.b), N.ptr(st["queue"]),
                         *self._sorted_workspaces())
            launch_terms(Tc, cfg, self._n_sm)
        C, _ = contact_bsr(ee, None, pt, None, V, t, out=getattr(self, "_C", None), status=st["status"],
                           read_status=False)
        self._C = C
        S, A = st["S"], self.A
        N.call("ipcb_bsr_union", V, N.ptr(S.offsets), N.ptr(S.columns), N.ptr(C.offsets), N.ptr(C.columns),
               N.ptr(A.offsets), N.ptr(st["a_rows"]), N.ptr(A.columns), N.ptr(st["src_a"]), N.ptr(st["src_b"]), cap,
               N.ptr(A.nnz_dev), N.ptr(st["status"]), N.ptr(st["ws"]), st["ws"].numel(), s)
        N.call("ipcb_newton_values", int(self.dtype == torch.float64), N.ptr(A.nnz_dev), cap, N.ptr(st["a_rows"]),
               N.ptr(A.columns), N.ptr(st["src_a"]), N.ptr(st["src_b"]), N.ptr(st["g_off"]), N.ptr(st["g_idx"]),
               N.ptr(st["tet_vals"]), h2, N.ptr(st["diag"]), N.ptr(C.values), h2, N.ptr(A.values), s)
        r = st["graph_read"]
        r[0:1].copy_(ee.cnt, non_blocking=True)
        r[1:2].copy_(pt.cnt, non_blocking=True)
        r[2:3].copy_(st["status"], non_blocking=True)
        r[3:4].copy_(self._status, non_blocking=True)

    def _compute_A_graph(self) -> BsrMatrix:
        """compute_A replayed from one CUDA graph with one host read.  The
        first call (and any call after a list overflow, a row with too many
        contact columns or a union over capacity) runs the step-by-step path,
        which grows the lists and has the autotuner pick the terms schedule;
        the sequence is then captured for the buffers and schedule of the
        moment and replayed while they stay the same."""
        st = self._static
        g = getattr(self, "_A_graph", None)
        if g is not None and g[0] == self._A_graph_key():
            g[1].replay()
            torch.cuda.current_stream().synchronize()
            n_ee, n_pt, bst, qst = (int(v) for v in st["graph_read"])
            ee, pt = self.contacts_new, self.contacts_pt
            if n_ee <= ee.capacity and n_pt <= pt.capacity and not (bst & (4 | 16)):
                self.n_contacts, self.n_contacts_pt = n_ee, n_pt
                self.query_status = qst
                if qst & QUERY_FAILED:
                    warnings.warn(f"contact query ran out of its traversal bound (status {qst}): "
                                  "the candidate lists may be incomplete", RuntimeWarning, stacklevel=2)
                self.collision_hessian = self._C
                return self.A
            self._A_graph = None  # overflow: the step-by-step path grows and re-tunes
        A = self._compute_A_queue()
        n_ee, n_pt = self.n_contacts, self.n_contacts_pt
        cfg = self._tuner.best.get(str((int(self.dtype == torch.float64), bucket(n_ee + n_pt), bucket(self.n_tets))))
        if cfg is None:
            return A
        cap = self._graph_buffers()
        graph = torch.cuda.CUDAGraph()
        torch.cuda.synchronize()
        with N.no_collection(), torch.cuda.graph(graph):
            self._enqueue_A(cfg, cap)
        self._A_graph = (self._A_graph_key(), graph, cfg)
        # the capture recorded the launches without running them: run them now
        # so that this call's results are the graph's (same matrix as above)
        graph.replay()
        torch.cuda.current_stream().synchronize()
        self.collision_hessian = self._C
        return self.A

    def _A_graph_key(self):
        """The buffers a captured compute_A reads and writes (the schedule is
        kept as captured while they stay: a later workload bucket's choice
        would cost a recapture per change of bucket)."""
        st = self._static
        ee, pt, t = self.contacts_new, self.contacts_pt, self.collision_triplets
        return (ee.a1a2b1b2.data_ptr(), ee.capacity, pt.a1a2b1b2.data_ptr(), pt.capacity,
                None if t is None else t.rows.data_ptr(), None if self.A is None else self.A.values.data_ptr(),
                None if getattr(self, "_C", None) is None else self._C.values.data_ptr(),
                st.get("a_rows").data_ptr() if "a_rows" in st else None, self.states.x.data_ptr())

    def _compute_A_generic(self) -> BsrMatrix:
        """Per-term kernels, then one sort-based assembly of every triplet."""
        h2 = self.h * self.h
        V = self.soup.n_verts
        self.b.zero_()
        t = self._elastic
        N.call("ipcb_tet_hessian", self.material, int(self.dtype == torch.float64), N.ptr(self.states.x),
               N.ptr(self.tets), self.n_tets, N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, N.ptr(t.rows),
               N.ptr(t.cols), N.ptr(t.vals), N.ptr(self.b), N.stream_handle())
        self.compute_contact_hessian(detect=True, build_bsr=False)
        nc = 16 * (self.n_contacts + self.n_contacts_pt)
        ct = self.collision_triplets
        idx = torch.arange(V, dtype=torch.int32, device=self.device)
        eye = torch.eye(3, dtype=self.dtype, device=self.device)
        diag = self.mass.to(self.dtype)[:, None, None] * eye
        if bool(self.fixed.any()):
            diag = diag + (h2 * self.k_att) * self.fixed.to(self.dtype)[:, None, None] * eye
        rows = torch.cat([idx, t.rows, ct.rows[:nc]])
        cols = torch.cat([idx, t.cols, ct.cols[:nc]])
        vals = torch.cat([diag, t.vals * h2, ct.vals[:nc] * h2])
        self.A = bsr_from_triplets(V, V, rows, cols, vals, out=getattr(self, "A", None))
        return self.A

    # ------------------------------------------------ work-queue assembly
    def _static_pattern(self):
        """Pattern of M + h^2 K (diagonal + mesh connectivity), built once,
        with the map from every slot to the tet blocks that land on it."""
        dev = self.device
        V, nt = self.soup.n_verts, self.n_tets
        T = self.tets
        rows_t = T.repeat_interleave(4, dim=1).reshape(-1).contiguous()
        cols_t = T.repeat(1, 4).reshape(-1).contiguous()
        idx = torch.arange(V, dtype=torch.int32, device=dev)
        rows = torch.cat([idx, rows_t])
        cols = torch.cat([idx, cols_t])
        ones = torch.ones((rows.numel(), 3, 3), dtype=self.dtype, device=dev)
        S = bsr_from_triplets(V, V, rows, cols, ones)
        nnz = int(S.nnz_dev.item())
        slots = torch.empty(16 * nt, dtype=torch.int32, device=dev)
        N.call("ipcb_bsr_slots", V, N.ptr(S.offsets), N.ptr(S.columns), 16 * nt, N.ptr(rows_t), N.ptr(cols_t),
               N.ptr(slots), N.stream_handle())
        sl = slots.long()
        g_idx = torch.argsort(sl, stable=True).to(torch.int32)
        g_off = torch.zeros(nnz + 1, dtype=torch.int32, device=dev)
        g_off[1:] = torch.cumsum(torch.bincount(sl, minlength=nnz), 0).to(torch.int32)
        h2 = self.h * self.h
        diag = (self.mass + (h2 * self.k_att) * self.fixed.double()).to(self.dtype)
        self._static = dict(S=S, nnz=nnz, g_off=g_off, g_idx=g_idx, diag=diag, rows_t=rows_t, cols_t=cols_t,
                            tet_vals=torch.empty((16 * nt, 3, 3), dtype=self.dtype, device=dev),
                            queue=torch.zeros(1, dtype=torch.int32, device=dev),
                            status=torch.zeros(1, dtype=torch.int32, device=dev),
                            ws=torch.empty(N.size("ipcb_bsr_union_workspace", V), dtype=torch.uint8, device=dev))
        n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
        self._n_sm = n_sm
        self._tuner = Autotuner("terms", terms_candidates())

    def _sorted_workspaces(self):
        """Device workspaces of the class-sorted narrow phase, one per list."""
        self._ws_ee = hessian_workspace(self.contacts_new, getattr(self, "_ws_ee", None))
        self._ws_pt = hessian_workspace(self.contacts_pt, getattr(self, "_ws_pt", None))
        return N.ptr(self._ws_ee), N.ptr(self._ws_pt)

    def _launch_terms(self, cfg, Tc):
        s = N.stream_handle()
        if cfg[0] == "separate":
            n_ee, n_pt = self.n_contacts, self.n_contacts_pt
            t = self.collision_triplets
            kappa = float(self.contact_stiffness)
            if n_ee:
                self._ws_ee = hessian_workspace(self.contacts_new, getattr(self, "_ws_ee", None))
                contact_hessian_ee(None, self.soup, self.contacts_new, t, self.b, kappa, n=n_ee, ws=self._ws_ee)
            if n_pt:
                self._ws_pt = hessian_workspace(self.contacts_pt, getattr(self, "_ws_pt", None))
                contact_hessian_pt(None, self.soup, self.contacts_pt, t, self.b, n_ee, kappa, n=n_pt,
                                   ws=self._ws_pt)
            N.call("ipcb_tet_hessian", self.material, int(self.dtype == torch.float64), N.ptr(self.states.x),
                   N.ptr(self.tets), self.n_tets, N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, None, None,
                   N.ptr(self._static["tet_vals"]), N.ptr(self.b), s)
            return
        launch_terms(Tc, cfg, self._n_sm)

    def _compute_A_queue(self) -> BsrMatrix:
        """Contact detection, then one persistent launch for the contact
        records and the tets (ipcb_terms_launch), the contact BSR, and the
        union with the fixed elastic pattern with gathered values."""
        if self._static is None:
            self._static_pattern()
        st = self._static
        h2 = self.h * self.h
        V = self.soup.n_verts
        self.b.zero_()
        with self.profile_timer("detect collision"):
            self.detect_collision()
        n_ee, n_pt = self.n_contacts, self.n_contacts_pt
        nc = 16 * (n_ee + n_pt)
        if getattr(self, "collision_triplets", None) is None or self.collision_triplets.rows.shape[0] < nc:
            self.collision_triplets = Triplets.zeros(max(nc, 16), self.dtype, self.device)
        t = self.collision_triplets
        Tc = N.Terms(int(self.dtype == torch.float64), N.ptr(self.states.x), N.ptr(self.soup.xcs),
                     self.contacts_new.c_struct(), self.contacts_pt.c_struct(), float(self.contact_stiffness),
                     N.ptr(t.rows), N.ptr(t.cols), N.ptr(t.vals), N.ptr(t.mask), self.material, N.ptr(self.tets),
                     self.n_tets, N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, None, None, N.ptr(st["tet_vals"]),
                     N.ptr(self.b), N.ptr(st["queue"]), *self._sorted_workspaces())
        key = (int(self.dtype == torch.float64), bucket(n_ee + n_pt), bucket(self.n_tets))
        cfg = self._tuner.pick(key, lambda c: self._launch_terms(c, Tc), self.b.zero_)
        self._launch_terms(cfg, Tc)
        C, cst = contact_bsr(self.contacts_new, n_ee, self.contacts_pt, n_pt, V, t, out=getattr(self, "_C", None),
                             status=st["status"])
        self._C = C
        if cst & 4:  # a row with too many distinct contact columns: sort-based assembly
            idx = torch.arange(V, dtype=torch.int32, device=self.device)
            eye = torch.eye(3, dtype=self.dtype, device=self.device)
            rows = torch.cat([idx, st["rows_t"], t.rows[:nc]])
            cols = torch.cat([idx, st["cols_t"], t.cols[:nc]])
            vals = torch.cat([st["diag"][:, None, None] * eye, st["tet_vals"] * h2, t.vals[:nc] * h2])
            self.A = bsr_from_triplets(V, V, rows, cols, vals)
            return self.A
        S = st["S"]
        cap = st["nnz"] + max(int(C.nnz_dev.item()), 1)  # the union's size bound
        A = getattr(self, "A", None)
        if A is None or A.columns.shape[0] < cap or "a_rows" not in st or st["a_rows"].shape[0] < cap:
            cap = cap + cap // 4
            A = BsrMatrix(V, V, cap, self.dtype, self.device)
            for k in ("a_rows", "src_a", "src_b"):
                st[k] = torch.empty(cap, dtype=torch.int32, device=self.device)
        cap = min(A.columns.shape[0], st["a_rows"].shape[0])
        s = N.stream_handle()
        N.call("ipcb_bsr_union", V, N.ptr(S.offsets), N.ptr(S.columns), N.ptr(C.offsets), N.ptr(C.columns),
               N.ptr(A.offsets), N.ptr(st["a_rows"]), N.ptr(A.columns), N.ptr(st["src_a"]), N.ptr(st["src_b"]), cap,
               N.ptr(A.nnz_dev), N.ptr(st["status"]), N.ptr(st["ws"]), st["ws"].numel(), s)
        N.call("ipcb_newton_values", int(self.dtype == torch.float64), N.ptr(A.nnz_dev), cap, N.ptr(st["a_rows"]),
               N.ptr(A.columns), N.ptr(st["src_a"]), N.ptr(st["src_b"]), N.ptr(st["g_off"]), N.ptr(st["g_idx"]),
               N.ptr(st["tet_vals"]), h2, N.ptr(st["diag"]), N.ptr(C.values), h2, N.ptr(A.values), s)
        self.A = A
        self.collision_hessian = C
        return A

    def compute_rhs(self) -> torch.Tensor:
        """time_integrator_base.py:82-91,428-438: gradient of the total energy."""
        h2 = self.h * self.h
        x = self.states.x.double()
        g = -h2 * self.b.double() + self.mass[:, None] * (x - self.x_tilde())
        if bool(self.fixed.any()):
            g = g + (h2 * self.k_att) * self.fixed.double()[:, None] * (x - self.x_target.double())
        self.rhs = g.to(self.dtype)
        return self.rhs

    def _direct(self):
        if self.direct_solver is None:
            from .direct import DirectSolver

            self.direct_solver = DirectSolver("metis")
        return self.direct_solver

    def solve(self) -> torch.Tensor:
        """time_integrator_base.py:502-507: PCG to the relative residual
        ``tol`` within ``maxiter`` (falling back to the direct solve when it
        misses), or the direct solve alone (``solve_ldlt``, 470-500)."""
        if self.linear_solver == "direct":
            dx = self._direct()(self.A, self.rhs)
        else:
            if self.host_pcg:
                dx, its, rel = pcg(self.A, self.rhs, self.precond_factory(self.A), self.tol, self.maxiter)
            else:
                if self._precond is None or self._precond_age >= self.precond_refresh or \
                        getattr(self._precond, "kind", 0) == 0:
                    self._precond = self.device_precond(self.A)
                    self._precond_age = 0
                self._precond_age += 1
                x, its, rel, status = self.device_pcg.solve(self.A, self.rhs, self._precond, self.tol, self.maxiter)
                dx = x
                if status:
                    rel = float("nan")
                    if status & 1:  # p^T A p <= 0: A is indefinite, the Cholesky fallback cannot succeed
                        self.stats.direct_failures += 1
                        self.stats.pcg_iterations.append(its)
                        return self._set_dx(dx)
            self.stats.pcg_iterations.append(its)
            if not (rel <= self.tol) and self.direct_fallback:
                from .direct import DirectSolverError

                try:
                    dx = self._direct()(self.A, self.rhs)
                    self.stats.fallbacks += 1
                except DirectSolverError:
                    # the Cholesky stand-in needs a positive definite matrix; an
                    # indefinite one (unprojected elastic Hessian under
                    # compression) keeps the PCG iterate, as the reference's cg
                    # returns its last iterate; the line search then tests descent
                    self.stats.direct_failures += 1
        return self._set_dx(dx)

    def _set_dx(self, dx: torch.Tensor) -> torch.Tensor:
        """states.dx = dx, copied into the existing tensor when it fits, so
        the captured line-search graph (which holds its address) stays valid."""
        cur = self.states.dx
        if cur is not None and cur.shape == dx.shape and cur.dtype == dx.dtype and cur.device == dx.device:
            if cur.data_ptr() != dx.data_ptr():
                cur.copy_(dx)
            return cur
        self.states.dx = dx.clone()
        return self.states.dx

    def line_search(self) -> float:
        """time_integrator_base.py:514-546 with the CCD bound."""
        if self.line_search_mode == "device":
            return self._line_search_device()
        return self._line_search_host()

    def _line_search_host(self) -> float:
        """The reference's loop: energies and the accept test on the host."""
        self._lists_at_x = False
        x_tmp = self.states.x.clone()
        E0 = self.total_energy()
        refusals = self.ccd_refusals
        ub = self.collision_free_step(self.states.dx)
        if self.ccd_refusals != refusals:
            # a CCD query ran out of its bounds: its TOI is no bound, no step
            self.stats.ccd_refusals += 1
            self.stats.energies.append((E0, E0))
            return 0.0
        alpha = ub
        accepted = False
        E1 = math.inf
        eps = 1.1920928955078125e-7 if self.dtype == torch.float32 else 2.220446049250313e-16
        for _ in range(64):
            self.states.x.copy_(x_tmp - alpha * self.states.dx)
            E1 = self.total_energy()
            if math.isfinite(E1) and E1 < E0:
                accepted = True
                break
            alpha *= 0.5
            if alpha <= eps * max(1.0, ub):
                break
        if not accepted:
            self.states.x.copy_(x_tmp)
            alpha = 0.0
        self.stats.energies.append((E0, E1))
        return alpha

    # ------------------------------------------------- device line search
    def _energy_launches(self, acc: torch.Tensor, detect: bool = True):
        """Launches (no host reads, graph-capturable) that add the energy terms
        at the current x into acc: [0] elastic Psi, [1] barrier, [2] inertia +
        attachment.  Contact lists are refilled by the DCD (their counts stay
        on the device), or, with detect=False, taken as they are."""
        s = N.stream_handle()
        fp64 = int(self.dtype == torch.float64)
        kappa = float(self.contact_stiffness)
        if detect:
            self.update_bvh()
            self._launch_dcd("ee")
            if self.has_triangles:
                self._launch_dcd("pt")
        soup = self.soup.c_struct()
        base = acc.data_ptr()
        N.call("ipcb_contact_energy", 0, ctypes.byref(soup), ctypes.byref(self.contacts_new.c_struct()), -1, kappa,
               base + 8, s)
        if self.has_triangles:
            N.call("ipcb_contact_energy", 1, ctypes.byref(soup), ctypes.byref(self.contacts_pt.c_struct()), -1,
                   kappa, base + 8, s)
        N.call("ipcb_tet_energy", self.material, fp64, N.ptr(self.states.x), N.ptr(self.tets), self.n_tets,
               N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, base, s)
        ls = self._ls
        N.call("ipcb_ls_inertia", fp64, self.soup.n_verts, N.ptr(self.states.x), N.ptr(self.states.x0),
               N.ptr(self.states.xdot), ls["gravity"], self.h, N.ptr(self.mass),
               N.ptr(ls["fixed"]) if ls["any_fixed"] else None, N.ptr(self.x_target), self.k_att, base + 16, s)

    def _ccd_launches(self, dx: torch.Tensor):
        """collision_free_step without its read: the TOI stays in ccd_toi."""
        soup = self.soup.c_struct()
        s = N.stream_handle()
        pad = 1e-7
        N.call("ipcb_add_dx", ctypes.byref(soup), N.ptr(dx), N.ptr(self.ccd_x1), s)
        N.call("ipcb_swept_edge_aabbs", ctypes.byref(soup), N.ptr(self.ccd_x1), pad, N.ptr(self.ccd_edge_lower),
               N.ptr(self.ccd_edge_upper), s)
        self.ccd_edge_bvh.refit(self.ccd_edge_lower, self.ccd_edge_upper)
        self.ccd_toi.fill_(1.0)
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

    def _ls_buffers(self):
        if self._ls is None:
            dev = self.device
            self._ls = dict(
                x_tmp=torch.empty_like(self.states.x), acc=torch.zeros(3, dtype=torch.float64, device=dev),
                acc0=torch.zeros(3, dtype=torch.float64, device=dev),
                state=torch.zeros(ctypes.sizeof(N.LsState), dtype=torch.uint8, device=dev),
                host=torch.zeros(ctypes.sizeof(N.LsState), dtype=torch.uint8).pin_memory(),
                gravity=(ctypes.c_double * 3)(*self.gravity.double().cpu().tolist()),
                fixed=self.fixed.to(torch.uint8), any_fixed=bool(self.fixed.any()),
                stream=torch.cuda.Stream(device=dev), graph=None, key=None)
        return self._ls

    def _ls_key(self):
        return (self.states.x.data_ptr(), self.states.dx.data_ptr(), self.states.x0.data_ptr(),
                self.states.xdot.data_ptr(), self.contacts_new.a1a2b1b2.data_ptr(), self.contacts_new.capacity,
                self.contacts_pt.a1a2b1b2.data_ptr(), self.contacts_pt.capacity, self.x_target.data_ptr())

    def _ls_graph(self):
        """The WHILE graph of one trial, captured once per buffer set (on a
        side stream: the legacy default stream cannot be captured)."""
        ls = self._ls
        key = self._ls_key()
        if ls["graph"] is not None and ls["key"] == key:
            return ls["graph"]
        if ls["graph"] is not None:
            N.lib().ipcb_graph_destroy(ls["graph"])
            ls["graph"] = None
        fp64 = int(self.dtype == torch.float64)
        h2 = self.h * self.h
        side = ls["stream"]
        side.wait_stream(torch.cuda.current_stream())
        ctx, handle = ctypes.c_void_p(), ctypes.c_ulonglong()
        # keep the collector off while capturing, so no tensor freed by a
        # collection (its allocator may record or query events) touches the
        # capturing stream
        gc_was_on = gc.isenabled()
        gc.disable()
        try:
            self._capture_trial(side, ctx, handle, fp64, h2)
        finally:
            if gc_was_on:
                gc.enable()
        torch.cuda.current_stream().wait_stream(side)
        ls["graph"], ls["key"] = ctx, key
        return ctx

    def _capture_trial(self, side, ctx, handle, fp64, h2):
        ls = self._ls
        with torch.cuda.stream(side):
            s = N.stream_handle()
            N.call("ipcb_graph_while_begin", ctypes.byref(ctx), ctypes.byref(handle), s)
            body_ok = False
            try:
                N.call("ipcb_ls_trial", N.ptr(ls["state"]), fp64, self.soup.n_verts, N.ptr(ls["x_tmp"]),
                       N.ptr(self.states.dx), N.ptr(self.states.x), N.ptr(ls["acc"]), s)
                self._energy_launches(ls["acc"])
                # the accept kernel is what ends the loop: the body is complete only with it
                N.call("ipcb_ls_accept", N.ptr(ls["state"]), N.ptr(ls["acc"]), h2,
                       ctypes.byref(self.contacts_new.c_struct()), ctypes.byref(self.contacts_pt.c_struct()),
                       handle.value, s)
                body_ok = True
            finally:
                end_rc = N.lib().ipcb_graph_while_end(ctx, s)
                if not body_ok or end_rc != 0:
                    N.lib().ipcb_graph_destroy(ctx)
            if end_rc != 0:
                raise N.NativeError("ipcb_graph_while_end failed: " + (N.lib().ipcb_last_error() or b"").decode())

    def _line_search_device(self) -> float:
        """The reference's search (same E0, bound, halving and accept test)
        with the trial loop on the device: E0 and the CCD bound are launched,
        then the WHILE graph runs trials until one is accepted, and the state
        is read once.  A contact-list overflow during the search grows the
        lists and reruns it on the host."""
        ls = self._ls_buffers()
        fp64 = int(self.dtype == torch.float64)
        h2 = self.h * self.h
        s = N.stream_handle()
        ls["x_tmp"].copy_(self.states.x)
        if getattr(self, "_ls_cache", False):
            # inside a step, x is the point the previous search accepted: its
            # energy terms are the accepted trial's (as the ABD search caches E0)
            ls["acc0"].copy_(ls["acc"])
        else:
            # within newton_iteration, compute_A has just detected the contacts
            # at this x: E0 uses its lists (the reference detects again, with
            # the same result)
            fresh = getattr(self, "_lists_at_x", False)
            ls["acc0"].zero_()
            self._energy_launches(ls["acc0"], detect=not fresh)
        self._lists_at_x = False
        self._ccd_launches(self.states.dx)
        eps = 1.1920928955078125e-7 if self.dtype == torch.float32 else 2.220446049250313e-16
        N.call("ipcb_ls_begin", N.ptr(ls["state"]), N.ptr(self.ccd_toi), fp64, N.ptr(self._status),
               N.ptr(ls["acc0"]), h2, eps, 64,
               ctypes.byref(self.contacts_new.c_struct()), ctypes.byref(self.contacts_pt.c_struct()), s)
        graph = self._ls_graph()
        N.call("ipcb_graph_launch", graph, s)
        N.call("ipcb_ls_finish", N.ptr(ls["state"]), fp64, self.soup.n_verts, N.ptr(ls["x_tmp"]),
               N.ptr(self.states.x), s)
        ls["host"].copy_(ls["state"], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        st = N.LsState.from_buffer_copy(ls["host"].numpy().tobytes())
        if st.overflow:
            if st.max_ee > self.contacts_new.capacity:
                self._grow_contact_list(self.contacts_new, st.max_ee)
            if st.max_pt > self.contacts_pt.capacity:
                self._grow_contact_list(self.contacts_pt, st.max_pt, point_triangle=True)
            self.states.x.copy_(ls["x_tmp"])
            return self._line_search_host()
        self.query_status = st.refused
        if st.refused:
            # a CCD query ran out of its bounds: its TOI is no bound, no step
            self.ccd_refusals += 1
            self.stats.ccd_refusals += 1
        self.stats.energies.append((st.E0, st.E1))
        self.ls_trials = st.it
        self._ls_cache = bool(getattr(self, "_in_step", False) and st.accepted)
        return st.alpha_accepted if st.accepted else 0.0

    def __del__(self):
        ls = getattr(self, "_ls", None)
        if ls and ls.get("graph") is not None:
            try:
                N.lib().ipcb_graph_destroy(ls["graph"])
            except Exception:
                pass

    def newton_iteration(self) -> tuple[float, float]:
        """One iteration of RodBCBase.step; with ``self.timing`` set, the
        device time of each phase (ms) is left in ``self.phase_ms``."""
        ev = None
        if getattr(self, "timing", False):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            ev[0].record()
        self.compute_A()
        if ev:
            ev[1].record()
        self.compute_rhs()
        if ev:
            ev[2].record()
        self.solve()
        if ev:
            ev[3].record()
        self._lists_at_x = True  # nothing has moved x since compute_A's detection
        alpha = self.line_search()
        if ev:
            ev[4].record()
            torch.cuda.synchronize()
            self.phase_ms = {k: ev[i].elapsed_time(ev[i + 1]) for i, k in
                             enumerate(("compute_A", "rhs", "solve", "line_search"))}
        norm = float(self.states.dx.double().abs().max()) if alpha > 0 else 0.0
        return alpha, norm

    def step(self) -> StepStats:
        """time_integrator_base.py:375-401."""
        self.stats = StepStats()
        self._precond = None  # a fresh factor at the first iteration of every step
        if self.boundary is not None:
            self.x_target.copy_(torch.as_tensor(self.boundary(self.time + self.h), dtype=self.dtype))
        # the line search may reuse the energy of the point it accepted last
        # only between iterations of this step (x~ and the targets are fixed)
        self._in_step, self._ls_cache = True, False
        try:
            for it in range(self.max_newton):
                alpha, norm = self.newton_iteration()
                self.stats.newton_iterations = it + 1
                self.stats.alphas.append(alpha)
                self.stats.norms.append(norm)
                if alpha == 0.0 or norm <= self.vel_tol * self.h:
                    break
        finally:
            self._in_step, self._ls_cache = False, False
        x = self.states.x
        self.states.xdot.copy_((x - self.states.x0) / self.h)
        self.states.x0.copy_(x)
        self.frame += 1
        self.time += self.h
        return self.stats
