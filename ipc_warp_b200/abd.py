"""Affine body dynamics on the IPC contact pipeline: ``AffineBodyDynamics``
and ``FixedBVHAffineBodyDynamics`` of the reference
(affine_body_dynamics.py:220-697, fixed_bvh_contacts.py:830-862) on the
sm_100a kernels of ipcb_abd_* (csrc/abd.cu).

Each body has four vec3 unknowns ``[p, a0, a1, a2]`` (``abd_states.q``,
shape (4 nb, 3)) and a surface vertex is x = p + r0 a0 + r1 a1 + r2 a2 with
r its body-local rest position (``xcs``: the world position at rest minus
the body's volume centroid).  One Newton iteration (``RodBCBase.step``,
time_integrator_base.py:375-401):

* ``compute_A``: contact detection, the vertex contact force and 16 Hessian
  blocks per record (ipcb_contact_hessian), then the reduced 12 nb system:
  ``assembly="direct"`` (default) builds the block pattern from the touching
  body pairs and folds every record into it (ipcb_abd_pattern +
  ipcb_abd_assemble); ``assembly="triplets"`` runs the reference pipeline
  (body triplets + 16x fan-out + sort/merge into BSR, affine_body_dynamics.py
  427-505).  Both give the same matrix.
* ``solve``: "cg" = device PCG (block Jacobi, relative residual 1e-4, 100
  iterations; the reference's warp cg) with the direct solve as fallback,
  "ldlt" = the direct sparse Cholesky (the reference's cuDSS LDLT).
* ``line_search``: CCD bound, then halving from it until the incremental
  potential (inertia + orthogonality + h^2 barrier, double) decreases, with
  the reference's energy caching (affine_body_dynamics.py:600-646).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from . import contact as contact_mod
from .bsr import BsrMatrix, Triplets, bsr_from_triplets
from .contact import ContactSolverBase, Soup
from .dynamic_contacts import ContactBarrierMixin
from .fixed_bvh_contacts import FixedBodyContactSolver
from .newton import DevicePcg, JacobiPrecond, StepStats


@dataclass
class ABDState:
    """affine_body_dynamics.py:33-39: (4 nb, 3) tensors."""
    q: torch.Tensor
    q0: torch.Tensor
    q_tilde: torch.Tensor
    qdot: torch.Tensor
    dx: torch.Tensor


@dataclass
class VertexStates:
    """The vertex state the contact code reads: x (= soup.x_transformed), x0, dx."""
    x: torch.Tensor
    x0: torch.Tensor
    dx: torch.Tensor


def mass_properties(vertices: np.ndarray, faces: np.ndarray, body: np.ndarray):
    """affine_body_dynamics.py:318-342: per body the volume centroid and
    |volume| of its closed surface (divergence theorem), per vertex a third
    of the area of every incident triangle."""
    nb = int(body.max()) + 1
    centers = np.zeros((nb, 3))
    volumes = np.zeros(nb)
    weights = np.zeros(len(vertices))
    fb_all = faces.reshape(-1, 3)
    fbody = body[fb_all[:, 0]]
    for b in range(nb):
        fb = fb_all[fbody == b]
        if len(fb) == 0:
            centers[b] = vertices[body == b].mean(axis=0)
            volumes[b] = 1.0
            weights[body == b] = 1.0
            continue
        a, c, d = vertices[fb[:, 0]], vertices[fb[:, 1]], vertices[fb[:, 2]]
        signed = np.einsum("ij,ij->i", a, np.cross(c, d)) / 6.0
        total = float(signed.sum())
        if abs(total) > 1e-12:
            centers[b] = (signed[:, None] * (a + c + d) / 4.0).sum(axis=0) / total
            volumes[b] = abs(total)
        else:
            centers[b] = vertices[body == b].mean(axis=0)
            volumes[b] = max(float(np.prod(np.ptp(vertices[body == b], axis=0))), 1e-12)
        area = 0.5 * np.linalg.norm(np.cross(c - a, d - a), axis=1)
        np.add.at(weights, fb.reshape(-1), np.repeat(area / 3.0, 3))
    return centers, volumes, weights


def mass_moments(local: np.ndarray, body: np.ndarray, weights: np.ndarray, volumes: np.ndarray,
                 density: float) -> np.ndarray:
    """affine_body_dynamics.py:344-358 as scalar moments (nb, 4, 4):
    sum_v w_v [1, r_v]^T [1, r_v], weights scaled to density * volume."""
    nb = len(volumes)
    M = np.zeros((nb, 4, 4))
    for b in range(nb):
        ids = np.flatnonzero(body == b)
        w = weights[ids]
        m = density * float(volumes[b])
        w = np.full(len(ids), m / len(ids)) if w.sum() == 0 else w / w.sum() * m
        C = np.column_stack((np.ones(len(ids)), local[ids]))
        M[b] = C.T @ (w[:, None] * C)
    return M


def _load_mesh(m):
    if isinstance(m, (tuple, list)) and len(m) == 2:
        v, f = m
        return np.asarray(v, np.float64), np.asarray(f, np.int64).reshape(-1, 3)
    raise TypeError("meshes are (vertices (n, 3), faces (m, 3)) pairs; mesh files are not read here")


def _edges(tris: np.ndarray) -> np.ndarray:
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    return np.unique(np.sort(e, axis=1), axis=0)


class AffineBodyDynamics(ContactBarrierMixin):
    """affine_body_dynamics.py:220-697 on the GPU."""

    def __init__(self, h, meshes, transforms=None, fixed_bodies=None, density=1000.0, affine_stiffness=1.0e8,
                 gravity=(0.0, 0.0, 0.0), motors=None, linear_solver=None, contact_kappa=None, *,
                 dhat: float = 1e-3, dtype=torch.float32, device="cuda", assembly: str = "direct",
                 velocity_tolerance: float = 5e-2, max_newton_iterations: int = 100, direct_fallback: bool = True):
        self.h = float(h)
        self.dtype = dtype
        self.device = torch.device(device)
        self.fp64 = int(dtype == torch.float64)
        if assembly not in ("direct", "triplets"):
            raise ValueError(f"unknown assembly {assembly!r}")
        self.assembly = assembly
        self.linear_solver = linear_solver or "cg"
        if self.linear_solver not in ("cg", "ldlt"):
            raise ValueError(f"Unknown ABD linear solver: {self.linear_solver!r}")
        self.direct_fallback = direct_fallback
        self.velocity_tolerance = float(velocity_tolerance)
        self.max_newton_iterations = int(max_newton_iterations)
        contact_mod._thickness = 0.5 * dhat
        contact_mod.buffer = 0.5 * dhat
        self.contact_stiffness = float(contact_kappa) if contact_kappa is not None else 1e9

        # geometry: world positions of every mesh under its transform
        if transforms is None:
            transforms = [np.eye(4) for _ in meshes]
        xs, fs, bs = [], [], []
        off = 0
        for b, (m, T) in enumerate(zip(meshes, transforms)):
            v, f = _load_mesh(m)
            T = np.asarray(T, np.float64)
            xs.append(v @ T[:3, :3].T + T[:3, 3])
            fs.append(f + off)
            bs.append(np.full(len(v), b, np.int32))
            off += len(v)
        world = np.concatenate(xs)
        faces = np.concatenate(fs)
        body = np.concatenate(bs)
        self.F = faces
        self.n_bodies = len(meshes)
        self.n_nodes = len(world)
        centers, volumes, weights = mass_properties(world, faces, body)
        local = world - centers[body]
        edges = _edges(faces)
        self.soup = Soup.from_numpy(world, edges.reshape(-1), faces.reshape(-1), body, xcs=local,
                                    device=self.device, dtype=dtype)
        self.xcs = self.soup.xcs
        self.body = self.soup.body
        x = self.soup.x_transformed
        self.states = VertexStates(x=x, x0=x.clone(), dx=torch.zeros_like(x))

        nb = self.n_bodies
        z = lambda: torch.zeros((4 * nb, 3), dtype=dtype, device=self.device)
        q = np.zeros((nb, 4, 3))
        q[:, 0] = centers
        q[:, 1:] = np.eye(3)
        self.abd_states = ABDState(q=z(), q0=z(), q_tilde=z(), qdot=z(), dx=z())
        self.abd_states.q.copy_(torch.tensor(q.reshape(-1, 3), dtype=dtype))
        self.abd_states.q0.copy_(self.abd_states.q)
        fixed = np.array([int(b in set(fixed_bodies or [])) for b in range(nb)], np.int32)
        self.abd_fixed = torch.tensor(fixed, device=self.device)
        self.abd_volume = torch.tensor(volumes, dtype=dtype, device=self.device)
        stiff = np.broadcast_to(np.asarray(affine_stiffness, np.float64), (nb,)).copy()
        self.abd_stiffness = torch.tensor(stiff, dtype=dtype, device=self.device)
        self.abd_mass = torch.tensor(mass_moments(local, body, weights, volumes, density).reshape(nb, 16),
                                     dtype=dtype, device=self.device)
        self.gravity = np.asarray(gravity, np.float64)
        omega = np.zeros((nb, 3))
        enabled = np.zeros(nb, np.int32)
        for b, w in (motors or {}).items():
            omega[int(b)] = w
            enabled[int(b)] = 1
        self.motor_omega = torch.tensor(omega, dtype=dtype, device=self.device)
        self.motor_enabled = torch.tensor(enabled, device=self.device)
        self._c_abd = N.Abd(nb, self.fp64, N.ptr(self.abd_states.q), N.ptr(self.abd_states.q0),
                            N.ptr(self.abd_states.q_tilde), N.ptr(self.abd_states.qdot), N.ptr(self.abd_states.dx),
                            N.ptr(self.abd_mass), N.ptr(self.abd_volume), N.ptr(self.abd_stiffness),
                            N.ptr(self.abd_fixed))

        self.reduced_b = z()
        self.reduced_contact_force = z()
        self.vertex_contact_force = torch.zeros_like(x)
        self.b = self.vertex_contact_force  # the contact kernels accumulate the vertex force here
        self._abd_status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._energy_acc = torch.zeros(2, dtype=torch.float64, device=self.device)
        self._pattern_ws = torch.empty(max(N.size("ipcb_abd_pattern_workspace", nb), 1), dtype=torch.uint8,
                                       device=self.device)
        self.body_off = torch.zeros(nb + 1, dtype=torch.int32, device=self.device)
        self.body_cols = torch.zeros(0, dtype=torch.int32, device=self.device)
        self.A = None
        self._body_triplets = None
        self.device_pcg = DevicePcg()
        self._dinv = None
        self.direct_solver = None
        self.stats = StepStats()
        self._cached_line_search_energy = None
        self._cached_state_potential_energy = None
        self._last_evaluated_potential_energy = None
        self.line_search_energy_cache_hits = 0
        self.line_search_potential_cache_hits = 0
        self.line_search_energy_evaluations = 0
        self.theta = 0.0
        self.frame = 0

        self._init_contacts()
        self.disable_self_collision = True
        self._sync_vertices()
        self._prepare_prediction()

    def _init_contacts(self):
        ContactSolverBase.__init__(self)

    # -------------------------------------------------------- small kernels
    def _sync_vertices(self):
        """affine_body_dynamics.py:360-362."""
        N.call("ipcb_abd_map", self.fp64, self.n_nodes, N.ptr(self.abd_states.q), N.ptr(self.xcs), N.ptr(self.body),
               N.ptr(self.states.x), N.stream_handle())

    def _vertex_direction(self):
        N.call("ipcb_abd_map", self.fp64, self.n_nodes, N.ptr(self.abd_states.dx), N.ptr(self.xcs),
               N.ptr(self.body), N.ptr(self.states.dx), N.stream_handle())

    def _prepare_prediction(self):
        g = (ctypes.c_double * 3)(*self.gravity)
        N.call("ipcb_abd_prepare_tilde", ctypes.byref(self._c_abd), self.h, g, N.ptr(self.motor_omega),
               N.ptr(self.motor_enabled), N.stream_handle())

    def set_initial_velocity(self, body=0, linear=(0.0, 0.0, 0.0), angular=(0.0, 0.0, 0.0)):
        """affine_body_dynamics.py:368-376: p_dot = v, a_j_dot = w x a_j."""
        o = 4 * int(body)
        q = self.abd_states.q[o:o + 4].double().cpu().numpy()
        qd = np.zeros((4, 3))
        qd[0] = linear
        w = np.asarray(angular, np.float64)
        for j in range(3):
            qd[1 + j] = np.cross(w, q[1 + j])
        self.abd_states.qdot[o:o + 4].copy_(torch.tensor(qd, dtype=self.dtype))

    def reset(self):
        self.abd_states.q.copy_(self.abd_states.q0)
        self.abd_states.qdot.zero_()
        self.abd_states.dx.zero_()
        self._cached_line_search_energy = None
        self._cached_state_potential_energy = None
        self._sync_vertices()
        self.theta = 0.0
        self.frame = 0

    def compute_V(self, ret=True):
        """affine_body_dynamics.py:685-691: vertices follow q."""
        self._sync_vertices()
        if ret:
            self.V = self.states.x.cpu().numpy()
            return self.V
        return None

    # --------------------------------------------------------------- system
    def _contact_blocks(self):
        """Detection, then the vertex force and 16 blocks per contact record."""
        self.vertex_contact_force.zero_()
        self.compute_contact_hessian(detect=True, build_bsr=False)
        return self.n_contacts, self.n_contacts_pt

    def compute_A(self) -> BsrMatrix:
        """affine_body_dynamics.py:427-505."""
        n_ee, n_pt = self._contact_blocks()
        if self.assembly == "triplets":
            return self._compute_A_triplets(n_ee, n_pt)
        nb = self.n_bodies
        n_rec = n_ee + n_pt
        t = self.collision_triplets
        pair_cap = nb + 2 * min(n_rec, nb * (nb - 1) // 2)
        if self.body_cols.numel() < pair_cap:
            self.body_cols = torch.zeros(pair_cap, dtype=torch.int32, device=self.device)
        cap = 16 * self.body_cols.numel()
        if self.A is None or self.A.values.shape[0] < cap:
            self.A = BsrMatrix(4 * nb, 4 * nb, cap, self.dtype, self.device)
        A = self.A
        s = N.stream_handle()
        self._abd_status.zero_()
        N.call("ipcb_abd_pattern", nb, N.ptr(self.abd_fixed), N.ptr(self.body), n_rec, N.ptr(t.rows), N.ptr(t.cols),
               N.ptr(t.mask), N.ptr(self.body_off), N.ptr(self.body_cols), self.body_cols.numel(), N.ptr(A.offsets),
               N.ptr(A.columns), N.ptr(A.nnz_dev), N.ptr(self._abd_status), N.ptr(self._pattern_ws),
               self._pattern_ws.numel(), s)
        N.call("ipcb_abd_assemble", ctypes.byref(self._c_abd), self.h * self.h, n_rec, n_ee, N.ptr(t.rows),
               N.ptr(t.cols), N.ptr(t.vals), N.ptr(t.mask), N.ptr(self.xcs), N.ptr(self.body), N.ptr(self.body_off),
               N.ptr(self.body_cols), N.ptr(A.offsets), N.ptr(A.nnz_dev), A.values.shape[0], N.ptr(A.values),
               N.ptr(self.reduced_b), self.n_nodes, N.ptr(self.vertex_contact_force),
               N.ptr(self.reduced_contact_force), N.ptr(self._abd_status), s)
        st = int(self._abd_status.item())
        if st:
            raise RuntimeError(f"ABD assembly status {st:#x} (a contact record spans more than two bodies)")
        self.collision_hessian = A
        self.b_reduced = self.reduced_b
        return A

    def _compute_A_triplets(self, n_ee, n_pt) -> BsrMatrix:
        """The reference pipeline: 16 body triplets per body, 16 reduced
        triplets per vertex block, then sort/merge into BSR."""
        nb = self.n_bodies
        h2 = self.h * self.h
        s = N.stream_handle()
        if self._body_triplets is None:
            self._body_triplets = Triplets.zeros(16 * nb, self.dtype, self.device)
        bt = self._body_triplets
        N.call("ipcb_abd_body_system", ctypes.byref(self._c_abd), h2, N.ptr(bt.rows), N.ptr(bt.cols),
               N.ptr(bt.vals), N.ptr(self.reduced_b), s)
        self.reduced_contact_force.zero_()
        N.call("ipcb_abd_reduce_force", ctypes.byref(self._c_abd), self.n_nodes, N.ptr(self.vertex_contact_force),
               N.ptr(self.xcs), N.ptr(self.body), N.ptr(self.reduced_contact_force), s)
        N.call("ipcb_abd_add_contact_gradient", self.fp64, 12 * nb, N.ptr(self.reduced_b),
               N.ptr(self.reduced_contact_force), h2, s)
        n_src = 16 * (n_ee + n_pt)
        rows, cols, vals = [bt.rows], [bt.cols], [bt.vals]
        if n_src:
            t = self.collision_triplets
            red = Triplets.zeros(16 * n_src, self.dtype, self.device)
            N.call("ipcb_abd_reduce_hessian", ctypes.byref(self._c_abd), n_src, N.ptr(t.rows), N.ptr(t.cols),
                   N.ptr(t.vals), N.ptr(self.xcs), N.ptr(self.body), h2, N.ptr(red.rows), N.ptr(red.cols),
                   N.ptr(red.vals), s)
            rows.append(red.rows)
            cols.append(red.cols)
            vals.append(red.vals)
        self.A = bsr_from_triplets(4 * nb, 4 * nb, torch.cat(rows), torch.cat(cols), torch.cat(vals))
        self.collision_hessian = self.A
        return self.A

    def compute_rhs(self):
        """compute_A assembles the reduced gradient (affine_body_dynamics.py:507-509)."""
        return self.reduced_b

    # ---------------------------------------------------------------- solve
    def _direct(self):
        if self.direct_solver is None:
            from .direct import DirectSolver

            self.direct_solver = DirectSolver("metis")
        return self.direct_solver

    def solve(self):
        """affine_body_dynamics.py:580-592."""
        if self.linear_solver == "ldlt":
            dq = self._direct()(self.A, self.reduced_b)
        else:
            M = JacobiPrecond(self.A, self._dinv)
            self._dinv = M.dinv
            x, its, rel, status = self.device_pcg.solve(self.A, self.reduced_b, M, 1e-4, 100)
            self.stats.pcg_iterations.append(its)
            dq = x
            if (status or not (rel <= 1e-4)) and self.direct_fallback:
                from .direct import DirectSolverError

                try:
                    dq = self._direct()(self.A, self.reduced_b)
                    self.stats.fallbacks += 1
                except DirectSolverError:  # indefinite: keep the PCG iterate
                    self.stats.direct_failures += 1
        self.abd_states.dx.copy_(dq)
        self._vertex_direction()
        return self.abd_states.dx

    # ---------------------------------------------------------- line search
    def _energies(self):
        """affine_body_dynamics.py:655-663: (inertia, orthogonality) in double."""
        self._energy_acc.zero_()
        N.call("ipcb_abd_body_energy", ctypes.byref(self._c_abd), self.h * self.h, N.ptr(self._energy_acc),
               N.stream_handle())
        e = self._energy_acc.cpu().numpy()
        return float(e[0]), float(e[1])

    def compute_inertia(self):
        return self._energies()[0]

    def compute_psi(self):
        return self._energies()[1]

    def compute_bc_energy(self):
        return 0.0

    def _compute_incremental_energy(self):
        self.line_search_energy_evaluations += 1
        inertia, ortho = self._energies()
        collision = self.compute_collision_energy()
        self._last_evaluated_potential_energy = ortho + collision
        return inertia + self._last_evaluated_potential_energy

    def line_search_upper_bound(self):
        self._vertex_direction()
        return self.collision_free_step(self.states.dx)

    def line_search(self):
        """affine_body_dynamics.py:600-646."""
        q_start = self.abd_states.q.clone()
        if self._cached_line_search_energy is None:
            if self._cached_state_potential_energy is None:
                e0 = self._compute_incremental_energy()
                e0_potential = self._last_evaluated_potential_energy
            else:
                inertia, _ = self._energies()
                e0_potential = self._cached_state_potential_energy
                e0 = inertia + e0_potential
                self.line_search_potential_cache_hits += 1
        else:
            e0 = self._cached_line_search_energy
            e0_potential = self._cached_state_potential_energy
            self.line_search_energy_cache_hits += 1
        upper = self.line_search_upper_bound()
        alpha = upper
        e1 = math.inf
        e1_potential = None
        accepted = False
        eps = 1.1920928955078125e-7 if self.dtype == torch.float32 else 2.220446049250313e-16
        s = N.stream_handle()
        for _ in range(64):
            N.call("ipcb_abd_step_from", self.fp64, 12 * self.n_bodies, N.ptr(q_start), N.ptr(self.abd_states.dx),
                   float(alpha), N.ptr(self.abd_states.q), s)
            self._sync_vertices()
            e1 = self._compute_incremental_energy()
            e1_potential = self._last_evaluated_potential_energy
            if math.isfinite(e1) and e1 < e0:
                accepted = True
                break
            alpha *= 0.5
            if alpha <= eps * max(1.0, upper):
                break
        if not accepted:
            self.abd_states.q.copy_(q_start)
            self._sync_vertices()
            alpha = 0.0
            self._cached_line_search_energy = e0
            self._cached_state_potential_energy = e0_potential
        else:
            self._cached_line_search_energy = e1
            self._cached_state_potential_energy = e1_potential
        self.stats.energies.append((e0, e1))
        return alpha

    # ----------------------------------------------------------------- step
    def update_x0_xdot(self):
        N.call("ipcb_abd_update_velocity", ctypes.byref(self._c_abd), self.h, N.stream_handle())
        self._sync_vertices()
        self.states.x0.copy_(self.states.x)

    def newton_iteration(self):
        self.compute_A()
        self.compute_rhs()
        self.solve()
        alpha = self.line_search()
        norm = float(self.states.dx.double().abs().max()) if alpha > 0 else 0.0
        return alpha, norm

    def step(self) -> StepStats:
        """affine_body_dynamics.py:378-384 + time_integrator_base.py:375-401."""
        self.stats = StepStats()
        self._prepare_prediction()
        self._cached_line_search_energy = None
        for it in range(self.max_newton_iterations):
            alpha, norm = self.newton_iteration()
            self.stats.newton_iterations = it + 1
            self.stats.alphas.append(alpha)
            self.stats.norms.append(norm)
            if alpha == 0.0 or not norm > self.velocity_tolerance * self.h:
                break
        self.update_x0_xdot()
        self.theta += self.h
        self.frame += 1
        return self.stats


class FixedBVHAffineBodyDynamics(AffineBodyDynamics, FixedBodyContactSolver):
    """fixed_bvh_contacts.py:830-862: ABD whose DCD/CCD query immutable
    body-local hierarchies (FixedBodyContactSolver)."""

    def _init_contacts(self):
        ContactSolverBase.__init__(self)
        self.initialize_fixed_body_bvhs(self.abd_states.q.view(-1))

    def detect_collision(self):
        return FixedBodyContactSolver.detect_collision(self)

    def collision_free_step(self, dx):
        return FixedBodyContactSolver.collision_free_step(self, dx)
