"""One Newton solve over deformable tets and affine bodies with IPC contact
(the batched affine + FEM wrecking-balls configuration).

The reference integrates tet bodies (``RodComplexBC``,
time_integrator_base.py:375-546 with fem/fem.py:139-203) and affine bodies
(``AffineBodyDynamics``, affine_body_dynamics.py:220-697) in separate
solvers.  Here both share one unknown vector ``q`` of vec3 entries -- the FEM
vertex positions, then p, a0, a1, a2 per affine body -- and one Newton
system:

* FEM part: lumped mass + h^2 tet Hessians (ipcb_tet_hessian), gradient
  M (x - x~) - h^2 f_elastic;
* affine part: the per-body inertia + orthogonality blocks and gradient
  (ipcb_abd_body_system), pendulum pins (ipcb_mixed_pins);
* contact: the vertex-space records (detect + ipcb_contact_hessian_sorted)
  reduced to J^T H J (ipcb_mixed_reduce_hessian) and -h^2 J^T f
  (ipcb_mixed_reduce_force); every triplet goes through one sort-based
  assembly (rows of a body collect all its contacts; ipcb_bsr_from_triplets
  handles such long rows with one CTA each).

The line search is the reference's backtracking (time_integrator_base.py
514-546) from the CCD bound of the vertex direction J dq, on the total
incremental potential in double.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _native as N
from . import contact as contact_mod
from .abd import mass_moments, mass_properties
from .bsr import BsrMatrix, Triplets, bsr_from_triplets
from .contact import Soup
from .autotune import Autotuner, bucket
from .dynamic_contacts import ContactBarrierMixin, hessian_workspace
from .newton import MATERIALS, DevicePcg, JacobiPrecond, StepStats, lame, launch_terms, terms_candidates
from .scenes import MixedScene


class MixedSolver(ContactBarrierMixin):
    """Tet FEM bodies + affine bodies + contact in one Newton solve."""

    def __init__(self, scene: MixedScene, *, material: str = "neo_hookean", E: float = 5e5, nu: float = 0.4,
                 rho: float = 1000.0, density: float = 1000.0, affine_stiffness: float = 1e8,
                 gravity=(0.0, -9.8, 0.0), h: float = 1e-2, dtype=torch.float32, device="cuda",
                 vel_tol: float = 5e-2, max_newton: int = 100, tol: float = 1e-4, maxiter: int = 500,
                 exclude_same_body: bool = True, direct_fallback: bool = True, assembly: str = "queue",
                 preconditioner: str = "body_block", line_search_mode: str = "device"):
        if assembly not in ("queue", "separate"):
            raise ValueError(f"unknown assembly {assembly!r}")
        if preconditioner not in ("body_block", "jacobi"):
            raise ValueError(f"unknown preconditioner {preconditioner!r}")
        self.assembly = assembly
        # "body_block": 3x3 blocks for the FEM vertices, the 12x12 diagonal
        # block for each affine body's (p, a0, a1, a2); "jacobi": 3x3 blocks
        # throughout
        self.preconditioner = preconditioner
        if line_search_mode not in ("device", "host"):
            raise ValueError(f"unknown line search mode {line_search_mode!r}")
        self.line_search_mode = line_search_mode
        self._ls = None
        self._acc_cached = False
        self._lists_at_q = False
        self.h = float(h)
        self.dtype = dtype
        self.device = torch.device(device)
        self.fp64 = int(dtype == torch.float64)
        self.material = MATERIALS[material]
        self.mu, self.lam = lame(E, nu)
        self.vel_tol, self.max_newton = float(vel_tol), int(max_newton)
        self.tol, self.maxiter = float(tol), int(maxiter)
        self.direct_fallback = direct_fallback
        self.contact_stiffness = float(scene.kappa)
        contact_mod._thickness = 0.5 * scene.dhat
        contact_mod.buffer = 0.5 * scene.dhat
        dev = self.device

        # ---- vertices: FEM first, then the affine bodies' surfaces
        fem = scene.fem
        Vf = fem.n_verts
        nb = len(scene.bodies)
        bv, bf, bb = [], [], []
        off = Vf
        for b, (v, f) in enumerate(scene.bodies):
            bv.append(np.asarray(v, np.float64))
            bf.append(np.asarray(f, np.int64).reshape(-1, 3) + off)
            bb.append(np.full(len(v), b, np.int32))
            off += len(v)
        world_a = np.concatenate(bv) if bv else np.zeros((0, 3))
        faces_a = np.concatenate(bf) if bf else np.zeros((0, 3), np.int64)
        body_a = np.concatenate(bb) if bb else np.zeros(0, np.int32)
        fixed = np.zeros(nb, np.int32)
        fixed[list(scene.fixed_bodies)] = 1
        # body volume centroids and moments (affine_body_dynamics.py:318-358)
        centers, volumes, weights = mass_properties(world_a, faces_a - Vf, body_a)
        local = world_a - centers[body_a]
        x = np.concatenate([fem.x, world_a])
        xcs = np.concatenate([fem.xcs, local])
        tris_a = faces_a.reshape(-1)
        e = np.concatenate([faces_a[:, [0, 1]], faces_a[:, [1, 2]], faces_a[:, [2, 0]]])
        edges_a = np.unique(np.sort(e, axis=1), axis=0).reshape(-1)
        n_fem_bodies = int(fem.body.max()) + 1 if Vf else 0
        soup_body = np.concatenate([fem.body, body_a + n_fem_bodies]).astype(np.int32)
        self.soup = Soup.from_numpy(x, np.concatenate([fem.edges, edges_a]).astype(np.int32),
                                    np.concatenate([fem.triangles, tris_a]).astype(np.int32), soup_body, xcs=xcs,
                                    device=dev, dtype=dtype)
        self.n_fem, self.n_bodies, self.n_verts = Vf, nb, x.shape[0]
        self.nq = Vf + 4 * nb
        self.F = np.concatenate([fem.triangles.reshape(-1, 3), faces_a])

        # ---- unknowns
        q = np.zeros((self.nq, 3))
        q[:Vf] = fem.x
        qa = np.zeros((nb, 4, 3))
        qa[:, 0] = centers
        qa[:, 1:] = np.eye(3)
        q[Vf:] = qa.reshape(-1, 3)
        z = lambda n: torch.zeros((n, 3), dtype=dtype, device=dev)  # noqa: E731
        self.q = torch.tensor(q, dtype=dtype, device=dev)
        self.dq = z(self.nq)
        self.q_start = z(self.nq)
        self.x = self.soup.x_transformed
        self.dx = torch.zeros_like(self.x)

        class _S:  # the contact code reads states.x / states.dx
            pass

        self.states = _S()
        self.states.x, self.states.dx = self.x, self.dx

        # ---- FEM state
        self.tets = torch.as_tensor(fem.tets, dtype=torch.int32, device=dev).contiguous()
        self.n_tets = self.tets.shape[0]
        self.Bm = torch.zeros((self.n_tets, 3, 3), dtype=dtype, device=dev)
        self.W = torch.zeros(self.n_tets, dtype=dtype, device=dev)
        if self.n_tets:
            N.call("ipcb_tet_rest", self.fp64, N.ptr(self.soup.xcs), N.ptr(self.tets), self.n_tets, N.ptr(self.Bm),
                   N.ptr(self.W), N.stream_handle())
        w = self.W.double().cpu().numpy()
        m = np.zeros(Vf)
        np.add.at(m, fem.tets.reshape(-1), np.repeat(rho * w / 4.0, 4))
        m[m == 0] = rho * (w.mean() if len(w) else 1.0) / 4.0
        self.fem_mass = torch.tensor(m, dtype=torch.float64, device=dev)
        self.gravity = np.asarray(gravity, np.float64)
        self.g_fem = torch.tensor(self.gravity, dtype=torch.float64, device=dev)
        self.x0_f = self.q[:Vf].clone()
        self.v_f = z(Vf)
        self.xt_f = torch.zeros((Vf, 3), dtype=torch.float64, device=dev)

        # ---- affine state (views of q / dq for the body range)
        self.qa = self.q[Vf:]
        self.q0_a = self.qa.clone()
        self.qt_a = z(4 * nb)
        self.qdot_a = z(4 * nb)
        for b, (lin, ang) in (scene.velocities or {}).items():
            o = 4 * int(b)
            qd = np.zeros((4, 3))
            qd[0] = lin
            for j in range(3):
                qd[1 + j] = np.cross(np.asarray(ang, np.float64), qa[int(b), 1 + j])
            self.qdot_a[o:o + 4] = torch.tensor(qd, dtype=dtype)
        self.abd_fixed = torch.tensor(fixed, device=dev)
        self.abd_volume = torch.tensor(volumes, dtype=dtype, device=dev)
        self.abd_stiffness = torch.full((nb,), float(affine_stiffness), dtype=dtype, device=dev)
        self.abd_mass = torch.tensor(mass_moments(local, body_a, weights, volumes, density).reshape(nb, 16),
                                     dtype=dtype, device=dev)
        self._c_abd = N.Abd(nb, self.fp64, N.ptr(self.qa), N.ptr(self.q0_a), N.ptr(self.qt_a), N.ptr(self.qdot_a),
                            N.ptr(self.dq[Vf:]), N.ptr(self.abd_mass), N.ptr(self.abd_volume),
                            N.ptr(self.abd_stiffness), N.ptr(self.abd_fixed))
        self.body_local = torch.tensor(body_a, dtype=torch.int32, device=dev)
        self._c_mixed = N.Mixed(self.fp64, Vf, self.n_verts, nb, N.ptr(self.body_local), N.ptr(self.abd_fixed),
                                N.ptr(self.soup.xcs))
        # pins: body-local point, world target, stiffness
        pr, pt, pk = np.zeros((nb, 3)), np.zeros((nb, 3)), np.zeros(nb)
        for b, (point, target, k) in (scene.pins or {}).items():
            pr[int(b)] = np.asarray(point, np.float64) - centers[int(b)]
            pt[int(b)] = target
            pk[int(b)] = k
        self.pin_rest = torch.tensor(pr, dtype=dtype, device=dev)
        self.pin_target = torch.tensor(pt, dtype=dtype, device=dev)
        self.pin_k = torch.tensor(pk, dtype=dtype, device=dev)

        # ---- buffers
        self.b = torch.zeros_like(self.x)  # vertex force (elastic + contact), -gradient
        self.rhs = z(self.nq)
        self._tet = Triplets.zeros(16 * self.n_tets, dtype, dev)
        self._body = Triplets.zeros(16 * nb, dtype, dev)
        self._pin = Triplets.zeros(16 * nb, dtype, dev)
        # the blocks of the fixed pattern in one array (tets | bodies | pins),
        # so one gather map covers them all
        nt16 = 16 * self.n_tets
        self._fixed_vals = torch.zeros((nt16 + 32 * nb, 3, 3), dtype=dtype, device=dev)
        self._tet.vals = self._fixed_vals[:nt16]
        self._body.vals = self._fixed_vals[nt16:nt16 + 16 * nb]
        self._pin.vals = self._fixed_vals[nt16 + 16 * nb:]
        # assemble A as the union of the fixed pattern (FEM mass, tets, body
        # blocks, pins; its slot map built once) and the reduced contact
        # blocks, instead of sorting every triplet each iteration
        self.fixed_pattern = True
        self._static = None
        self._red = None
        self._red_ws = None
        self._red_n = torch.zeros(1, dtype=torch.int32, device=dev)
        self._status = torch.zeros(1, dtype=torch.int32, device=dev)
        self._acc = torch.zeros(4, dtype=torch.float64, device=dev)
        self._queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self._n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
        self._tuner = Autotuner("mixed_terms", terms_candidates())
        self.A = None
        self.device_pcg = DevicePcg()
        self._dinv = None
        self._dinv_group = None
        self._in_step, self._E_cache = False, None
        self.direct_solver = None
        self.stats = StepStats()
        self.frame = 0
        self.time = 0.0

        ContactBarrierMixin.__init__(self)
        self.disable_self_collision = exclude_same_body
        self._sync()
        self.prepare()

    # ------------------------------------------------------------- maps
    def _sync(self):
        """x = J q for every soup vertex."""
        self._lists_at_q = False  # q may have moved: the contact lists are not known to be current
        N.call("ipcb_mixed_map", ctypes.byref(self._c_mixed), N.ptr(self.q), N.ptr(self.x), N.stream_handle())

    def _vertex_direction(self):
        N.call("ipcb_mixed_map", ctypes.byref(self._c_mixed), N.ptr(self.dq), N.ptr(self.dx), N.stream_handle())

    def prepare(self):
        """Predictors: x~ = x0 + h v + h^2 g (FEM), q~ of the affine bodies
        (affine_body_dynamics.py:378-384)."""
        h = self.h
        self.xt_f.copy_(self.x0_f.double() + h * self.v_f.double() + h * h * self.g_fem)
        g = (ctypes.c_double * 3)(*self.gravity)
        if self.n_bodies:
            N.call("ipcb_abd_prepare_tilde", ctypes.byref(self._c_abd), h, g, None, None, N.stream_handle())

    # ----------------------------------------------------------- system
    def _reduced_contact(self, n_rec: int, h2: float) -> Triplets:
        """J^T H J of the contact records' triplets, scaled by h^2."""
        n_src = 16 * n_rec
        if n_src == 0:
            return None
        t = self.collision_triplets
        need = N.size("ipcb_mixed_hessian_workspace", n_src)
        if self._red_ws is None or self._red_ws.numel() < need:
            self._red_ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        for _ in range(2):
            cap = 0 if self._red is None else self._red.rows.shape[0]
            self._status.zero_()
            N.call("ipcb_mixed_reduce_hessian", ctypes.byref(self._c_mixed), n_src, N.ptr(t.rows), N.ptr(t.cols),
                   N.ptr(t.vals), N.ptr(t.mask), h2, cap, N.ptr(self._red.rows) if cap else None,
                   N.ptr(self._red.cols) if cap else None, N.ptr(self._red.vals) if cap else None,
                   N.ptr(self._red_n), N.ptr(self._status), N.ptr(self._red_ws), self._red_ws.numel(),
                   N.stream_handle())
            n = int(self._red_n.item())
            if n == 0:
                return None
            if n <= cap:
                return Triplets(self._red.rows[:n], self._red.cols[:n], self._red.vals[:n])
            self._red = Triplets.zeros(n + n // 4 + 16, self.dtype, self.device)
        raise RuntimeError("mixed contact reduction did not fit its grown capacity")

    def _terms_struct(self, h2: float):
        """The persistent launch's view of this iteration: contact lists
        (class-sorted), tets and the affine bodies' (i, j) items."""
        t, tt, bt = self.collision_triplets, self._tet, self._body
        self._ws_ee = hessian_workspace(self.contacts_new, getattr(self, "_ws_ee", None))
        self._ws_pt = hessian_workspace(self.contacts_pt, getattr(self, "_ws_pt", None))
        Tc = N.Terms(self.fp64, N.ptr(self.x), N.ptr(self.soup.xcs), self.contacts_new.c_struct(),
                     self.contacts_pt.c_struct(), float(self.contact_stiffness), N.ptr(t.rows), N.ptr(t.cols),
                     N.ptr(t.vals), N.ptr(t.mask), self.material, N.ptr(self.tets), self.n_tets, N.ptr(self.Bm),
                     N.ptr(self.W), self.mu, self.lam, N.ptr(tt.rows), N.ptr(tt.cols), N.ptr(tt.vals), N.ptr(self.b),
                     N.ptr(self._queue), N.ptr(self._ws_ee), N.ptr(self._ws_pt))
        Tc.abd = self._c_abd
        Tc.body_row0, Tc.h2 = self.n_fem, h2
        Tc.a_rows, Tc.a_cols, Tc.a_vals = N.ptr(bt.rows), N.ptr(bt.cols), N.ptr(bt.vals)
        Tc.a_grad = N.ptr(self.rhs[self.n_fem:])
        return Tc

    def _terms_separate(self, h2: float):
        """The per-kind kernels: tets, class-sorted EE / PT, body system."""
        s = N.stream_handle()
        if self.n_tets:
            t = self._tet
            N.call("ipcb_tet_hessian", self.material, self.fp64, N.ptr(self.x), N.ptr(self.tets), self.n_tets,
                   N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, N.ptr(t.rows), N.ptr(t.cols), N.ptr(t.vals),
                   N.ptr(self.b), s)
        self.compute_contact_hessian(detect=False, build_bsr=False)
        if self.n_bodies:
            bt = self._body
            N.call("ipcb_abd_body_system", ctypes.byref(self._c_abd), h2, N.ptr(bt.rows), N.ptr(bt.cols),
                   N.ptr(bt.vals), N.ptr(self.rhs[self.n_fem:]), s)
            bt.rows.add_(self.n_fem)  # body-local rows -> unknown rows
            bt.cols.add_(self.n_fem)

    def _run_terms(self, cfg, Tc, h2):
        if cfg[0] == "separate":
            self._terms_separate(h2)
        else:
            launch_terms(Tc, cfg, self._n_sm)

    def compute_A(self) -> BsrMatrix:
        """The Newton matrix and gradient at q: FEM mass + h^2 tets, affine
        bodies + pins, and the reduced contact Hessian; gradient in self.rhs.
        The per-iteration terms run as one persistent launch or as per-kind
        kernels, whichever the autotuner measured faster for this workload
        (``assembly="queue"``), or always per kind (``"separate"``)."""
        h2 = self.h * self.h
        Vf, nb = self.n_fem, self.n_bodies
        s = N.stream_handle()
        self.b.zero_()
        if self._lists_at_q:
            # the search that produced q evaluated its energy here: its
            # detection (hierarchies refit, lists filled at q) is this one
            self.n_contacts, self.n_contacts_pt = (
                int(v) for v in torch.cat([self.contacts_new.cnt, self.contacts_pt.cnt]).tolist())
        else:
            with self.profile_timer("detect collision"):
                self.detect_collision()
        n_ee, n_pt = self.n_contacts, self.n_contacts_pt
        n_rec = n_ee + n_pt
        if getattr(self, "collision_triplets", None) is None or self.collision_triplets.rows.shape[0] < 16 * n_rec:
            self.collision_triplets = Triplets.zeros(max(16 * n_rec, 16), self.dtype, self.device)
        # gradient: FEM inertia, body inertia + orthogonality (written by the
        # terms), pins, -h^2 J^T b
        g = self.rhs
        g[:Vf] = (self.fem_mass[:, None] * (self.q[:Vf].double() - self.xt_f)).to(self.dtype)
        if self.assembly == "separate":
            self._terms_separate(h2)
        else:
            Tc = self._terms_struct(h2)
            key = (self.fp64, bucket(n_rec), bucket(self.n_tets), nb)
            cfg = self._tuner.pick(key, lambda c: self._run_terms(c, Tc, h2), self.b.zero_)
            self._run_terms(cfg, Tc, h2)
        if nb:
            pt = self._pin
            N.call("ipcb_mixed_pins", ctypes.byref(self._c_mixed), N.ptr(self.q), N.ptr(self.pin_rest),
                   N.ptr(self.pin_target), N.ptr(self.pin_k), h2, N.ptr(pt.rows), N.ptr(pt.cols), N.ptr(pt.vals),
                   N.ptr(g), None, s)
        N.call("ipcb_mixed_reduce_force", ctypes.byref(self._c_mixed), N.ptr(self.b), -h2, N.ptr(g), s)
        red = self._reduced_contact(n_rec, h2)
        if self.fixed_pattern:
            return self._assemble_union(red, h2)
        idx = torch.arange(Vf, dtype=torch.int32, device=self.device)
        eye = torch.eye(3, dtype=self.dtype, device=self.device)
        rows, cols, vals = [idx], [idx], [self.fem_mass.to(self.dtype)[:, None, None] * eye]
        if self.n_tets:
            rows.append(self._tet.rows)
            cols.append(self._tet.cols)
            vals.append(self._tet.vals * h2)
        if nb:
            for tr in (self._body, self._pin):
                rows.append(tr.rows)
                cols.append(tr.cols)
                vals.append(tr.vals)
        if red is not None:
            rows.append(red.rows)
            cols.append(red.cols)
            vals.append(red.vals)
        self.A = bsr_from_triplets(self.nq, self.nq, torch.cat(rows), torch.cat(cols), torch.cat(vals), out=self.A)
        return self.A

    def _static_pattern(self):
        """Pattern of FEM mass + tets + body blocks + pins (their rows and
        columns are the same every iteration) with the map from each slot to
        the blocks of _fixed_vals that land on it, built once."""
        dev = self.device
        Vf, nb, nt16 = self.n_fem, self.n_bodies, 16 * self.n_tets
        rows_g = torch.cat([self._tet.rows, self._body.rows, self._pin.rows])
        cols_g = torch.cat([self._tet.cols, self._body.cols, self._pin.cols])
        idx = torch.arange(self.nq, dtype=torch.int32, device=dev)
        rows = torch.cat([idx, rows_g])
        cols = torch.cat([idx, cols_g])
        ones = torch.ones((rows.numel(), 3, 3), dtype=self.dtype, device=dev)
        S = bsr_from_triplets(self.nq, self.nq, rows, cols, ones)
        nnz = int(S.nnz_dev.item())
        n_g = rows_g.numel()
        slots = torch.empty(max(n_g, 1), dtype=torch.int32, device=dev)
        N.call("ipcb_bsr_slots", self.nq, N.ptr(S.offsets), N.ptr(S.columns), n_g, N.ptr(rows_g), N.ptr(cols_g),
               N.ptr(slots), N.stream_handle())
        sl = slots[:n_g].long()
        g_idx = torch.argsort(sl, stable=True).to(torch.int32)
        g_off = torch.zeros(nnz + 1, dtype=torch.int32, device=dev)
        g_off[1:] = torch.cumsum(torch.bincount(sl, minlength=nnz), 0).to(torch.int32)
        diag = torch.zeros(self.nq, dtype=self.dtype, device=dev)
        diag[:Vf] = self.fem_mass.to(self.dtype)
        self._static = dict(S=S, nnz=nnz, g_off=g_off, g_idx=g_idx, diag=diag, n_fixed=nt16,
                            status=torch.zeros(1, dtype=torch.int32, device=dev),
                            ws=torch.empty(N.size("ipcb_bsr_union_workspace", self.nq), dtype=torch.uint8,
                                           device=dev))

    def _assemble_union(self, red, h2: float) -> BsrMatrix:
        """A = union of the fixed pattern (values gathered in a fixed order:
        h^2 times the tet blocks, the body and pin blocks, the FEM mass on
        the diagonal) and the BSR of the reduced contact triplets."""
        if self._static is None:
            self._static_pattern()
        st = self._static
        s = N.stream_handle()
        # ipcb_newton_values scales every gathered block by h^2: the body and
        # pin blocks (unscaled terms) enter divided by it
        self._fixed_vals[st["n_fixed"]:].mul_(1.0 / h2)
        if red is None:
            red = Triplets.zeros(1, self.dtype, self.device)  # one zero block at (0, 0)
            n = 1
        else:
            n = red.rows.shape[0]
        C = bsr_from_triplets(self.nq, self.nq, red.rows, red.cols, red.vals, count=n,
                              out=getattr(self, "_C", None))
        self._C = C
        S = st["S"]
        cap = st["nnz"] + max(int(C.nnz_dev.item()), 1)
        A = self.A
        if A is None or A.columns.shape[0] < cap or "a_rows" not in st or st["a_rows"].shape[0] < cap:
            cap = cap + cap // 4
            A = BsrMatrix(self.nq, self.nq, cap, self.dtype, self.device)
            for k in ("a_rows", "src_a", "src_b"):
                st[k] = torch.empty(cap, dtype=torch.int32, device=self.device)
        cap = min(A.columns.shape[0], st["a_rows"].shape[0])
        N.call("ipcb_bsr_union", self.nq, N.ptr(S.offsets), N.ptr(S.columns), N.ptr(C.offsets), N.ptr(C.columns),
               N.ptr(A.offsets), N.ptr(st["a_rows"]), N.ptr(A.columns), N.ptr(st["src_a"]), N.ptr(st["src_b"]), cap,
               N.ptr(A.nnz_dev), N.ptr(st["status"]), N.ptr(st["ws"]), st["ws"].numel(), s)
        N.call("ipcb_newton_values", self.fp64, N.ptr(A.nnz_dev), cap, N.ptr(st["a_rows"]), N.ptr(A.columns),
               N.ptr(st["src_a"]), N.ptr(st["src_b"]), N.ptr(st["g_off"]), N.ptr(st["g_idx"]),
               N.ptr(self._fixed_vals), h2, N.ptr(st["diag"]), N.ptr(C.values), 1.0, N.ptr(A.values), s)
        self.A = A
        return A

    def compute_rhs(self) -> torch.Tensor:
        return self.rhs

    # ------------------------------------------------------------ solve
    def _direct(self):
        if self.direct_solver is None:
            from .direct import DirectSolver

            self.direct_solver = DirectSolver("metis")
        return self.direct_solver

    def solve(self) -> torch.Tensor:
        """Block-Jacobi PCG to the relative residual ``tol`` (device loop),
        the direct solve as fallback when it misses (time_integrator_base.py
        502-507)."""
        groups = (self.n_fem, self.n_bodies) if self.preconditioner == "body_block" and self.n_bodies else None
        M = JacobiPrecond(self.A, self._dinv, groups=groups, out_group=self._dinv_group)
        self._dinv, self._dinv_group = M.dinv, M.dinv_group
        x, its, rel, status = self.device_pcg.solve(self.A, self.rhs, M, self.tol, self.maxiter)
        self.stats.pcg_iterations.append(its)
        dq = x
        if (status or not (rel <= self.tol)) and self.direct_fallback:
            from .direct import DirectSolverError

            try:
                dq = self._direct()(self.A, self.rhs)
                self.stats.fallbacks += 1
            except DirectSolverError:
                self.stats.direct_failures += 1
        self.dq.copy_(dq)
        self._vertex_direction()
        return self.dq

    # ------------------------------------------------------ line search
    def total_energy(self) -> float:
        """h^2 Psi_tets + FEM inertia + body inertia + h^2 orthogonality +
        pins + h^2 barrier at the current q (double)."""
        h2 = self.h * self.h
        acc = self._acc.zero_()
        s = N.stream_handle()
        if self.n_tets:
            N.call("ipcb_tet_energy", self.material, self.fp64, N.ptr(self.x), N.ptr(self.tets), self.n_tets,
                   N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, N.ptr(acc[0:1]), s)
        if self.n_bodies:
            N.call("ipcb_abd_body_energy", ctypes.byref(self._c_abd), h2, N.ptr(acc[1:3]), s)
            N.call("ipcb_mixed_pins", ctypes.byref(self._c_mixed), N.ptr(self.q), N.ptr(self.pin_rest),
                   N.ptr(self.pin_target), N.ptr(self.pin_k), h2, None, None, None, None, N.ptr(acc[3:4]), s)
        d = self.q[:self.n_fem].double() - self.xt_f
        inertia_f = 0.5 * (self.fem_mass[:, None] * d * d).sum()
        e = acc.cpu().numpy()
        return h2 * float(e[0]) + float(e[1]) + float(e[2]) + float(e[3]) + float(inertia_f) + \
            self.compute_collision_energy()

    def line_search(self) -> float:
        """Backtracking from the CCD bound on the total incremental potential
        (time_integrator_base.py:514-546): on the device ("device", the
        trials in one WHILE-graph launch, one host read) or on the host."""
        if self.line_search_mode == "device":
            return self._line_search_device()
        return self._line_search_host()

    # ---- device search: the FEM solver's ipcb_ls_* state machine over q
    def _ls_buffers(self):
        if self._ls is None:
            dev = self.device
            z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
            self._ls = dict(acc=z(3), acc0=z(3), extra=z(4),
                            state=torch.zeros(ctypes.sizeof(N.LsState), dtype=torch.uint8, device=dev),
                            host=torch.zeros(ctypes.sizeof(N.LsState), dtype=torch.uint8).pin_memory(),
                            gravity=(ctypes.c_double * 3)(*self.gravity),
                            stream=torch.cuda.Stream(device=dev), graph=None, key=None)
        return self._ls

    def _energy_launches(self, acc: torch.Tensor, detect: bool = True):
        """Launches (no host read) adding the energy at the current q into
        acc: [0] tet Psi, [1] barrier (both times h^2 in E), [2] FEM and body
        inertia, h^2 orthogonality and pins -- the terms of total_energy.  The
        contact lists are refilled by the DCD, their counts kept on the
        device."""
        s = N.stream_handle()
        h2 = self.h * self.h
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
        if self.n_tets:
            N.call("ipcb_tet_energy", self.material, self.fp64, N.ptr(self.x), N.ptr(self.tets), self.n_tets,
                   N.ptr(self.Bm), N.ptr(self.W), self.mu, self.lam, base, s)
        ls = self._ls
        eb = ls["extra"].data_ptr()
        if self.n_bodies:
            N.call("ipcb_abd_body_energy", ctypes.byref(self._c_abd), h2, eb, s)
            N.call("ipcb_mixed_pins", ctypes.byref(self._c_mixed), N.ptr(self.q), N.ptr(self.pin_rest),
                   N.ptr(self.pin_target), N.ptr(self.pin_k), h2, None, None, None, None, eb + 16, s)
        if self.n_fem:  # 1/2 m |q - x~|^2 with x~ = x0 + h v + h^2 g formed in double, as prepare() does
            N.call("ipcb_ls_inertia", self.fp64, self.n_fem, N.ptr(self.q), N.ptr(self.x0_f), N.ptr(self.v_f),
                   ls["gravity"], self.h, N.ptr(self.fem_mass), None, None, 0.0, eb + 24, s)
        N.call("ipcb_acc_fold", base + 16, eb, 4, s)

    def _ls_key(self):
        ee, pt = self.contacts_new, self.contacts_pt
        return (self.q.data_ptr(), self.q_start.data_ptr(), self.dq.data_ptr(), self.x.data_ptr(),
                ee.a1a2b1b2.data_ptr(), ee.capacity, pt.a1a2b1b2.data_ptr(), pt.capacity)

    def _ls_graph(self):
        """The WHILE graph of one trial (q = q_start - alpha dq, x = J q, the
        energy, the accept test), captured once per buffer set on a side
        stream."""
        ls = self._ls
        key = self._ls_key()
        if ls["graph"] is not None and ls["key"] == key:
            return ls["graph"]
        if ls["graph"] is not None:
            N.lib().ipcb_graph_destroy(ls["graph"])
            ls["graph"] = None
        h2 = self.h * self.h
        side = ls["stream"]
        side.wait_stream(torch.cuda.current_stream())
        ctx, handle = ctypes.c_void_p(), ctypes.c_ulonglong()
        with N.no_collection(), torch.cuda.stream(side):
            s = N.stream_handle()
            N.call("ipcb_graph_while_begin", ctypes.byref(ctx), ctypes.byref(handle), s)
            body_ok = False
            try:
                N.call("ipcb_ls_trial", N.ptr(ls["state"]), self.fp64, self.nq, N.ptr(self.q_start), N.ptr(self.dq),
                       N.ptr(self.q), N.ptr(ls["acc"]), s)
                self._sync()
                self._energy_launches(ls["acc"])
                # the accept kernel ends the body: it sets the loop condition
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
        torch.cuda.current_stream().wait_stream(side)
        ls["graph"], ls["key"] = ctx, key
        return ctx

    def _line_search_device(self) -> float:
        """E0 (inside step(): the terms of the point the previous search
        ended at) and the CCD bound are launched, the WHILE graph runs the
        trials, and the state is read once.  A contact list that overflows
        during the search grows and the search reruns on the host."""
        ls = self._ls_buffers()
        h2 = self.h * self.h
        s = N.stream_handle()
        self.q_start.copy_(self.q)
        if self._in_step and self._acc_cached:
            ls["acc0"].copy_(ls["acc"])
        else:
            ls["acc0"].zero_()
            self._energy_launches(ls["acc0"])
        self._launch_ccd(self.dx)
        eps = 1.1920928955078125e-7 if self.dtype == torch.float32 else 2.220446049250313e-16
        N.call("ipcb_ls_begin", N.ptr(ls["state"]), N.ptr(self.ccd_toi), self.fp64, N.ptr(self._status),
               N.ptr(ls["acc0"]), h2, eps, 64, ctypes.byref(self.contacts_new.c_struct()),
               ctypes.byref(self.contacts_pt.c_struct()), s)
        N.call("ipcb_graph_launch", self._ls_graph(), s)
        N.call("ipcb_ls_finish", N.ptr(ls["state"]), self.fp64, self.nq, N.ptr(self.q_start), N.ptr(self.q), s)
        self._sync()
        ls["host"].copy_(ls["state"], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        st = N.LsState.from_buffer_copy(ls["host"].numpy().tobytes())
        if st.overflow:
            if st.max_ee > self.contacts_new.capacity:
                self._grow_contact_list(self.contacts_new, st.max_ee)
            if st.max_pt > self.contacts_pt.capacity:
                self._grow_contact_list(self.contacts_pt, st.max_pt, point_triangle=True)
            self.q.copy_(self.q_start)
            self._sync()
            self._acc_cached = False
            return self._line_search_host()
        self.query_status = st.refused
        if st.refused:  # a CCD query ran out of its bounds: its TOI is no bound, no step
            self.ccd_refusals += 1
            self.stats.ccd_refusals += 1
        if not st.accepted:  # q is back at q_start: its terms are E0's
            ls["acc"].copy_(ls["acc0"])
        self._acc_cached = True
        # the accepted trial, the last one run, detected the contacts at q
        self._lists_at_q = bool(st.accepted)
        self.stats.energies.append((st.E0, st.E1))
        return st.alpha_accepted if st.accepted else 0.0

    def __del__(self):
        ls = getattr(self, "_ls", None)
        if ls and ls.get("graph") is not None:
            try:
                N.lib().ipcb_graph_destroy(ls["graph"])
            except Exception:
                pass

    def _line_search_host(self) -> float:
        """Inside step(), E0 is the energy of the point the previous search
        ended at (q has not moved since), as the reference's affine-body
        search caches it; a search outside step() evaluates it."""
        self.q_start.copy_(self.q)
        cached = self._E_cache if self._in_step else None
        E0 = cached if cached is not None else self.total_energy()
        self._E_cache = E0
        refusals = self.ccd_refusals
        ub = self.collision_free_step(self.dx)
        if self.ccd_refusals != refusals:
            self.stats.ccd_refusals += 1
            self.stats.energies.append((E0, E0))
            return 0.0
        alpha = ub
        eps = 1.1920928955078125e-7 if self.dtype == torch.float32 else 2.220446049250313e-16
        accepted, E1 = False, math.inf
        s = N.stream_handle()
        for _ in range(64):
            N.call("ipcb_abd_step_from", self.fp64, 3 * self.nq, N.ptr(self.q_start), N.ptr(self.dq), float(alpha),
                   N.ptr(self.q), s)
            self._sync()
            E1 = self.total_energy()
            if math.isfinite(E1) and E1 < E0:
                accepted = True
                break
            alpha *= 0.5
            if alpha <= eps * max(1.0, ub):
                break
        if not accepted:
            self.q.copy_(self.q_start)
            self._sync()
            alpha = 0.0
        else:
            self._E_cache = E1
            self._lists_at_q = True  # total_energy at the accepted q detected its contacts
        self.stats.energies.append((E0, E1))
        return alpha

    # ------------------------------------------------------------- step
    def newton_iteration(self) -> tuple[float, float]:
        self.compute_A()
        self.solve()
        alpha = self.line_search()
        norm = float(self.dx.double().abs().max()) if alpha > 0 else 0.0
        return alpha, norm

    def step(self) -> StepStats:
        """time_integrator_base.py:375-401 over the joint unknowns."""
        self.stats = StepStats()
        self.prepare()
        self._in_step, self._E_cache, self._acc_cached = True, None, False
        try:
            for it in range(self.max_newton):
                alpha, norm = self.newton_iteration()
                self.stats.newton_iterations = it + 1
                self.stats.alphas.append(alpha)
                self.stats.norms.append(norm)
                if alpha == 0.0 or norm <= self.vel_tol * self.h:
                    break
        finally:
            self._in_step, self._E_cache, self._acc_cached = False, None, False
        h = self.h
        Vf = self.n_fem
        self.v_f.copy_((self.q[:Vf] - self.x0_f) / h)
        self.x0_f.copy_(self.q[:Vf])
        if self.n_bodies:
            N.call("ipcb_abd_update_velocity", ctypes.byref(self._c_abd), h, N.stream_handle())
        self.frame += 1
        self.time += h
        return self.stats

    # ------------------------------------------------------------ checks
    def body_centres(self) -> np.ndarray:
        return self.qa.view(self.n_bodies, 4, 3)[:, 0].double().cpu().numpy()

    def orthogonality_error(self) -> float:
        """max over moving bodies of |A^T A - I| (screw_and_nut.py:38-62's
        check of an affine body staying rigid)."""
        A = self.qa.view(self.n_bodies, 4, 3)[:, 1:].double()
        moving = self.abd_fixed == 0
        if not bool(moving.any()):
            return 0.0
        G = A[moving] @ A[moving].transpose(1, 2)
        return float((G - torch.eye(3, dtype=G.dtype, device=G.device)).abs().max())
