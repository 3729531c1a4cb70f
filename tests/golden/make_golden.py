"""Generate golden vectors by running the reference's own hot-path functions.

The reference (ipc_warp) is Warp DSL code and its `ipctkwp` submodule is
empty, so it cannot be imported as is.  This script parses the reference
source files, takes the function and struct definitions of the contact path
by name, rewrites Warp's query loops (``while wp.bvh_query_next(q, j):`` into
``for j in q:``) and executes them as plain Python against
warp_standin.py.  The math that the reference imports from the missing
submodule is restated below (IPC barrier, EE mollifier, squared-distance
gradients and the negative spectral part of their Hessians) from Li et al.
2020, so what these vectors pin is the reference's own control flow:
closest-point regions, candidate filters and record order, cubic root
isolation, coplanarity polynomial, feature dispatch and Hessian composition.

Run in a container that has the reference checkout:

    python tests/golden/make_golden.py /path/to/ipc_warp

It writes tests/golden/*.npz.  Nothing at test time reads the reference.
"""
from __future__ import annotations

import ast
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import warp_standin as wp  # noqa: E402

wp.types = wp.types_


# ------------------------------------------------------------ source loader
class _QueryLoops(ast.NodeTransformer):
    """while wp.<x>_query_<...>next(q, j): body  ->  for j in q: body"""

    def visit_While(self, node):
        self.generic_visit(node)
        t = node.test
        if (isinstance(t, ast.Call) and isinstance(t.func, ast.Attribute) and t.func.attr.endswith("next")
                and len(t.args) == 2 and isinstance(t.args[1], ast.Name)):
            return ast.copy_location(
                ast.For(target=ast.Name(id=t.args[1].id, ctx=ast.Store()), iter=t.args[0], body=node.body,
                        orelse=[], type_comment=None), node)
        return node


def load(path: str, names, ns: dict, assigns=()):
    tree = ast.parse(open(path).read(), filename=path)
    keep = []
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)) and node.name in names:
            keep.append(node)
        elif isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in assigns for t in node.targets):
            keep.append(node)
    missing = set(names) - {n.name for n in keep if hasattr(n, "name")}
    assert not missing, (path, missing)
    mod = ast.Module(body=keep, type_ignores=[])
    mod = ast.fix_missing_locations(_QueryLoops().visit(mod))
    exec(compile(mod, path, "exec"), ns)
    return ns


def scalar_ns(fp64: bool) -> dict:
    """The names scalar_types.py defines, for either precision."""
    f = np.float64 if fp64 else np.float32
    ns = {"wp": wp, "np": np}
    ns.update(
        scalar=f, energy_scalar=f,
        vec2=wp._Vec(2, f), vec3=wp._Vec(3, f), vec4=wp._Vec(4, f),
        mat22=wp._Mat(2, 2, f), mat33=wp._Mat(3, 3, f), mat44=wp._Mat(4, 4, f),
        mat23=wp._Mat(2, 3, f), mat34=wp._Mat(3, 4, f), mat24=wp._Mat(2, 4, f),
        mat12=wp._Mat(12, 12, f), mat99=wp._Mat(9, 9, f), vec12=wp._Vec(12, f),
        scalar_epsilon=2.220446049250313e-16 if fp64 else 1.1920928955078125e-7,
    )
    return ns


# -------------------------------------- restated ipctkwp (Li et al. 2020)
def restated_ipc(ns: dict):
    f = ns["scalar"]

    def ipc_barrier(d2, d02, kappa):
        if d2 >= d02:
            return f(0)
        return f(-kappa * (d2 - d02) ** 2 * np.log(d2 / d02))

    def ipc_barrier_derivative(d2, d02, kappa):
        if d2 >= d02:
            return f(0)
        dx = d2 - d02
        return f(kappa * (-2 * dx * np.log(d2 / d02) - dx * dx / d2))

    def ipc_barrier_derivative2(d2, d02, kappa):
        if d2 >= d02:
            return f(0)
        dx = d2 - d02
        return f(kappa * (-2 * np.log(d2 / d02) - 4 * dx / d2 + dx * dx / (d2 * d2)))

    def ee_mollifier_threshold(x0, x1, x2, x3):
        ea, eb = x1 - x0, x3 - x2
        return f(1e-3) * wp.dot(ea, ea) * wp.dot(eb, eb)

    def _cross2(x0, x1, x2, x3):
        ea, eb = (x1 - x0).astype(np.float64), (x3 - x2).astype(np.float64)
        return ea, eb, float(np.dot(np.cross(ea, eb), np.cross(ea, eb)))

    def ee_mollifier_value(x0, x1, x2, x3, eps_x):
        _, _, xc = _cross2(x0, x1, x2, x3)
        if xc < eps_x:
            q = xc / eps_x
            return f((2 - q) * q)
        return f(1)

    def ee_mollifier_gradient_hessian_psd(x0, x1, x2, x3, eps_x):
        ea, eb, xc = _cross2(x0, x1, x2, x3)
        g = np.zeros(12)
        H = np.zeros((12, 12))
        if xc < eps_x:
            dm = 2 * (1 - xc / eps_x) / eps_x
            d2m = -2 / eps_x ** 2
            ab = ea.dot(eb)
            gxa = 2 * eb.dot(eb) * ea - 2 * ab * eb
            gxb = 2 * ea.dot(ea) * eb - 2 * ab * ea
            gx6 = np.concatenate([gxa, gxb])
            I3 = np.eye(3)
            Haa = 2 * eb.dot(eb) * I3 - 2 * np.outer(eb, eb)
            Hbb = 2 * ea.dot(ea) * I3 - 2 * np.outer(ea, ea)
            Hab = 4 * np.outer(ea, eb) - 2 * np.outer(eb, ea) - 2 * ab * I3
            H6 = d2m * np.outer(gx6, gx6) + dm * np.block([[Haa, Hab], [Hab.T, Hbb]])
            w, V = np.linalg.eigh(0.5 * (H6 + H6.T))
            H6 = (V * np.maximum(w, 0)) @ V.T
            L = np.zeros((6, 12))
            L[0:3, 0:3], L[0:3, 3:6] = -np.eye(3), np.eye(3)
            L[3:6, 6:9], L[3:6, 9:12] = -np.eye(3), np.eye(3)
            g = dm * (L.T @ gx6)
            H = L.T @ H6 @ L
        return g.astype(f), H.astype(f)

    def _param_dist(c, D, xs):
        """grad and NSD of min_tau |sum_k c_k(tau) x_k|^2 (c affine in tau)."""
        X = np.array(xs, dtype=np.float64)
        c = np.asarray(c, dtype=np.float64)
        D = np.asarray(D, dtype=np.float64).reshape(-1, len(c))
        r = c @ X
        E = D @ X
        G = 2 * E @ E.T
        n = len(c)
        B = np.zeros((3 * n, D.shape[0]))
        for j in range(D.shape[0]):
            B[:, j] = 2 * (np.kron(c, E[j]) + np.kron(D[j], r))
        H = 2 * np.kron(np.outer(c, c), np.eye(3)) - B @ np.linalg.solve(G, B.T)
        w, V = np.linalg.eigh(0.5 * (H + H.T))
        nsd = (V * np.minimum(w, 0)) @ V.T
        grad = 2 * np.kron(c, r)
        return grad, nsd

    def x_to_grad_nsd_hess_pt(x0, x1, x2, x3):
        X = [np.asarray(v, np.float64) for v in (x0, x1, x2, x3)]
        e1, e2, w = X[2] - X[1], X[3] - X[1], X[0] - X[1]
        A = np.array([[e1 @ e1, e1 @ e2], [e1 @ e2, e2 @ e2]])
        be, ga = np.linalg.solve(A, [e1 @ w, e2 @ w])
        g, h = _param_dist([1, -1 + be + ga, -be, -ga], [[0, 1, -1, 0], [0, 1, 0, -1]], X)
        return g.astype(f), h.astype(f)

    def x_to_grad_nsd_hess_ee(x0, x1, x2, x3):
        X = [np.asarray(v, np.float64) for v in (x0, x1, x2, x3)]
        ea, eb, w = X[1] - X[0], X[3] - X[2], X[0] - X[2]
        A = np.array([[ea @ ea, -ea @ eb], [-ea @ eb, eb @ eb]])
        s, t = np.linalg.solve(A, [-ea @ w, eb @ w])
        g, h = _param_dist([1 - s, s, -(1 - t), -t], [[-1, 1, 0, 0], [0, 0, 1, -1]], X)
        return g.astype(f), h.astype(f)

    def point_edge_distance_gradient_nsd_hessian(p, e0, e1):
        X = [np.asarray(v, np.float64) for v in (p, e0, e1)]
        e = X[2] - X[1]
        t = (X[0] - X[1]) @ e / (e @ e)
        g, h = _param_dist([1, -(1 - t), -t], [[0, 1, -1]], X)
        return g.reshape(3, 3).astype(f), h.astype(f)

    def beta_gamma_pt(x0, x1, x2, x3):
        e1, e2, w = x2 - x1, x3 - x1, x0 - x1
        a11, a12, a22, b1, b2 = e1 @ e1, e1 @ e2, e2 @ e2, e1 @ w, e2 @ w
        det = a11 * a22 - a12 * a12
        return (b1 * a22 - a12 * b2) / det, (a11 * b2 - a12 * b1) / det

    def beta_gamma_ee(x0, x1, x2, x3):
        ea, eb, w = x1 - x0, x3 - x2, x2 - x0
        a11, a12, a22, b1, b2 = ea @ ea, ea @ eb, eb @ eb, ea @ w, eb @ w
        det = a11 * a22 - a12 * a12
        return (b1 * a22 - a12 * b2) / det, (a11 * b2 - a12 * b1) / det

    ns.update({k: v for k, v in locals().items() if callable(v) and not k.startswith("_")})
    return ns


# ----------------------------------------------------------------- builders
def reference_ns(ref: str, fp64: bool) -> dict:
    ns = restated_ipc(scalar_ns(fp64))
    load(os.path.join(ref, "ccd", "cubic_roots.py"),
         ["evaluate", "multi_sign", "is_different_sign", "deflate", "find_closed", "quadratic_roots", "cubic_roots",
          "construct_3_root_polynomial", "construct_2_root_polynomial"], ns, assigns=("x_error",))
    load(os.path.join(ref, "ccd", "ccd.py"),
         ["verify_root_pt", "verify_root_ee", "build_and_solve_4_points_coplanar", "det_polynomial", "cubic_binomial",
          "pt_collision_time", "ee_collision_time", "swept_edge_aabbs", "swept_triangle_aabbs"], ns)
    load(os.path.join(ref, "contact.py"),
         ["edge_aabb", "XConstraint", "Contacts", "fetch_dist_v0v1", "fetch_dist_v0v1_pt", "_hash", "append",
          "edge_edge_collision", "closest_point_triangle", "point_triangle_collision"], ns,
         assigns=("_thickness", "buffer", "eps", "contact_volume"))
    load(os.path.join(ref, "dynamic_contacts.py"),
         ["embed_point_point_distance", "embed_point_edge_distance", "edge_edge_distance_gradient_hessian",
          "point_triangle_distance_gradient_hessian", "ee_mollifier_threshold_rest", "symmetric_outer_product_psd_12",
          "contact_hessian_ee", "contact_hessian_pt", "contact_energy_ee", "contact_energy_pt"], ns)
    return ns


def make_contacts(ns, capacity):
    c = ns["Contacts"]()
    c.list = [ns["XConstraint"](a1a2b1b2=None, e0e1=None, l0=None, alpha=None, lam=None) for _ in range(capacity)]
    c.cnt = np.zeros(1, np.int64)
    c.htable = np.full(8191, -1, np.int64)
    c.capacity = capacity
    return c


def records(c):
    n = int(c.cnt[0])
    return np.array([list(c.list[k].a1a2b1b2) + list(c.list[k].e0e1) for k in range(min(n, c.capacity))],
                    dtype=np.int32).reshape(-1, 6)


def run_dcd(ns, sc, x, exclude):
    """contact.py edge_aabb + edge_edge_collision + point_triangle_collision."""
    th = np.float32(sc.thickness)
    ns["_thickness"] = float(th)
    ns["buffer"] = float(th)
    soup = types.SimpleNamespace(edges=sc.edges, triangles=sc.triangles, body=sc.body, x_transformed=x, xcs=x)
    ne, nt = sc.n_edges, sc.n_tris
    lo, hi = np.zeros((ne, 3), np.float32), np.zeros((ne, 3), np.float32)
    wp.launch(ns["edge_aabb"], ne, x, sc.edges, lo, hi, ns["scalar"](th + th))
    ee = make_contacts(ns, 4096)
    wp.launch(ns["edge_edge_collision"], ne, wp.BoxSet(lo, hi), soup, ee, th, exclude)
    x32 = x.astype(np.float32)
    T = sc.triangles.reshape(-1, 3)
    tlo, thi = x32[T].min(axis=1), x32[T].max(axis=1)
    pt = make_contacts(ns, 4096)
    wp.launch(ns["point_triangle_collision"], sc.n_verts, wp.BoxSet(tlo, thi), soup, pt, th, exclude)
    return records(ee), records(pt), ee, pt


MATERIAL_FILES = {"snh": ("snh.py", ["reparam", "psi", "partialJpartialF", "PK1", "tangent_stiffness"]),
                  "neo_hookean": ("neo_hookean.py", ["tangent_stiffness", "PK1", "psi"]),
                  "stvk": ("stvk.py", ["tangent_stiffness", "psi", "PK1"])}


def fem_ns(ref: str, fp64: bool, material: str, mu: float, lam: float) -> dict:
    """fem/fem.py compute_Dm + tet_kernel_sparse and time_integrator_base.py
    compute_Psi over one material file (the reference selects the material
    by import, fem/fem.py:12-14); mu and lam as the material files read them
    from fem/params.py."""
    ns = scalar_ns(fp64)
    ns["mu"], ns["lam"] = ns["scalar"](mu), ns["scalar"](lam)
    fname, funcs = MATERIAL_FILES[material]
    load(os.path.join(ref, "fem", fname), funcs, ns)
    load(os.path.join(ref, "fem", "fem.py"), ["Triplets", "compute_Dm", "tet_kernel_sparse"], ns)
    load(os.path.join(ref, "time_integrator_base.py"), ["compute_Psi"], ns)
    return ns


def make_fem(ref: str):
    """F. tet terms (fem/fem.py:22-35,139-203, time_integrator_base.py:125-137)
    for the three materials in both builds, on a deformed 2x2x2-cell block."""
    from ipc_warp_b200 import scenes

    rng = np.random.default_rng(77)
    m = scenes.hex_grid_tets(2, 2, 2, size=(0.2, 0.2, 0.2))
    xcs = m.x.astype(np.float64)
    G = np.eye(3) + 0.12 * rng.normal(size=(3, 3))
    x = xcs @ G.T + 0.004 * rng.normal(size=xcs.shape)
    tets = m.tets.astype(np.int32)
    nt = len(tets)
    E_, nu = 1e5, 0.4
    mu, lam = E_ / (2 * (1 + nu)), E_ * nu / ((1 + nu) * (1 - 2 * nu))
    out = {"x": x, "xcs": xcs, "tets": tets, "mu": mu, "lam": lam}
    for material in MATERIAL_FILES:
        for fp64 in (True, False):
            ns = fem_ns(ref, fp64, material, mu, lam)
            f = ns["scalar"]
            xs, xr = x.astype(f), xcs.astype(f)
            geo = types.SimpleNamespace(xcs=xr, T=tets)
            Bm = np.zeros((nt, 3, 3), f)
            W = np.zeros(nt, f)
            wp.launch(ns["compute_Dm"], nt, geo, Bm, W)
            trip = types.SimpleNamespace(rows=np.zeros(16 * nt, np.int32), cols=np.zeros(16 * nt, np.int32),
                                         vals=np.zeros((16 * nt, 3, 3), f))
            b = np.zeros_like(xs)
            wp.launch(ns["tet_kernel_sparse"], 16 * nt, xs, geo, Bm, W, trip, b)
            Psi = np.zeros(nt, f)
            wp.launch(ns["compute_Psi"], nt, xs, geo, Bm, W, Psi)
            key = f"{material}_{64 if fp64 else 32}"
            out.update({f"{key}_rows": trip.rows, f"{key}_cols": trip.cols, f"{key}_vals": trip.vals,
                        f"{key}_force": b, f"{key}_psi": Psi, f"{key}_W": W})
    np.savez_compressed(os.path.join(HERE, "fem_tets.npz"), **out)


def make_abd(ref: str):
    """G. affine-body kernels (affine_body_dynamics.py:42-217) in both builds:
    body blocks and gradient, energies, and the vertex -> affine reductions of
    a contact force and of contact Hessian triplets."""
    rng = np.random.default_rng(78)
    nb = 3
    fixed = np.array([0, 0, 1], np.int32)
    nv_b = 7
    body = np.repeat(np.arange(nb), nv_b).astype(np.int32)
    rest = rng.normal(scale=0.3, size=(nb * nv_b, 3))
    q = np.zeros((nb, 4, 3))
    for b in range(nb):
        Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        A = Q @ (np.eye(3) + 0.05 * rng.normal(size=(3, 3)))
        q[b, 0] = rng.normal(size=3)
        q[b, 1:] = A.T  # columns a0, a1, a2
    qt = q + 0.01 * rng.normal(size=q.shape)
    L = rng.normal(size=(nb, 4, 4))
    M = np.einsum("bij,bkj->bik", L, L) + 4 * np.eye(4)  # SPD scalar moments
    volume = rng.uniform(0.5, 1.5, nb)
    stiffness = rng.uniform(1e3, 1e4, nb)
    h2 = 1e-4
    f_vert = rng.normal(size=(nb * nv_b, 3))
    n_src = 40
    src_rows = rng.integers(0, nb * nv_b, n_src).astype(np.int32)
    src_cols = rng.integers(0, nb * nv_b, n_src).astype(np.int32)
    src_vals = rng.normal(size=(n_src, 3, 3))
    out = {"q": q, "qt": qt, "M": M, "volume": volume, "stiffness": stiffness, "fixed": fixed, "h2": h2,
           "rest": rest, "body": body, "f_vert": f_vert, "src_rows": src_rows, "src_cols": src_cols,
           "src_vals": src_vals, "scale": 0.25}
    for fp64 in (True, False):
        ns = scalar_ns(fp64)
        f = ns["scalar"]
        load(os.path.join(ref, "affine_body_dynamics.py"),
             ["ABDState", "_assemble_body_system", "_reduce_contact_force", "_reduce_contact_hessian",
              "_body_energy"], ns)
        load(os.path.join(ref, "fem", "fem.py"), ["Triplets"], ns)
        st = types.SimpleNamespace(q=q.reshape(-1, 3).astype(f), q_tilde=qt.reshape(-1, 3).astype(f))
        mass = np.einsum("bij,kl->bijkl", M, np.eye(3)).reshape(-1, 3, 3).astype(f)
        trip = types.SimpleNamespace(rows=np.zeros(16 * nb, np.int32), cols=np.zeros(16 * nb, np.int32),
                                     vals=np.zeros((16 * nb, 3, 3), f))
        grad = np.zeros((4 * nb, 3), f)
        wp.launch(ns["_assemble_body_system"], 16 * nb, st, mass, volume.astype(f), stiffness.astype(f), fixed,
                  f(h2), trip, grad)
        inertia, ortho = np.zeros(1, f), np.zeros(1, f)
        wp.launch(ns["_body_energy"], nb, st, mass, volume.astype(f), stiffness.astype(f), fixed, f(h2), inertia,
                  ortho)
        red = np.zeros((4 * nb, 3), f)
        wp.launch(ns["_reduce_contact_force"], nb * nv_b, f_vert.astype(f), rest.astype(f), body, fixed, red)
        src = types.SimpleNamespace(rows=src_rows, cols=src_cols, vals=src_vals.astype(f))
        dst = types.SimpleNamespace(rows=np.zeros(16 * n_src, np.int32), cols=np.zeros(16 * n_src, np.int32),
                                    vals=np.zeros((16 * n_src, 3, 3), f))
        wp.launch(ns["_reduce_contact_hessian"], 16 * n_src, src, rest.astype(f), body, fixed, f(0.25), dst)
        key = "64" if fp64 else "32"
        out.update({f"rows_{key}": trip.rows, f"cols_{key}": trip.cols, f"vals_{key}": trip.vals,
                    f"grad_{key}": grad, f"inertia_{key}": inertia[0], f"ortho_{key}": ortho[0],
                    f"reduced_force_{key}": red, f"dst_rows_{key}": dst.rows, f"dst_cols_{key}": dst.cols,
                    f"dst_vals_{key}": dst.vals})
    np.savez_compressed(os.path.join(HERE, "abd_bodies.npz"), **out)


def make_fp32(ref: str):
    """H. the reference's float32 build (scalar_types.py:6, USE_FLOAT32) on the
    CCD path: per-pair collision times (ccd.py:304-357) and cubic roots
    (cubic_roots.py:96-193) evaluated in float32, beside the float64 build on
    the same float32 inputs.  Two sets of motions: the random ones of
    collision_time.npz, and near-contact motions of unit-scale geometry (a
    pair up to dhat = 1e-3 apart closing by 2 dhat), the configurations the
    scene CCD meets."""
    ns32 = reference_ns(ref, fp64=False)
    ns64 = reference_ns(ref, fp64=True)
    ct = np.load(os.path.join(HERE, "collision_time.npz"))
    rng = np.random.default_rng(79)
    sets = {}
    n = 1500
    sets["random"] = (ct["p0"][:n].astype(np.float32), ct["p1"][:n].astype(np.float32))
    # near contact at unit scale: 0.1-long edges / 0.1-wide triangles whose
    # centres lie in [-1, 1]^3, a pair placed up to dhat = 1e-3 apart along a
    # random normal and closing by 2 dhat (plus 0.2 dhat noise) over the step
    m = 2000
    c = rng.uniform(-1, 1, size=(m, 1, 3))
    nrm = rng.normal(size=(m, 1, 3))
    nrm /= np.linalg.norm(nrm, axis=2, keepdims=True)
    d0 = rng.uniform(0, 1e-3, size=(m, 1, 1))
    u = np.cross(nrm, rng.normal(size=(m, 1, 3)))
    u /= np.linalg.norm(u, axis=2, keepdims=True)
    v = np.cross(nrm, u)
    ang = rng.uniform(0, np.pi, size=(m, 1, 1))
    w = np.cos(ang) * u + np.sin(ang) * v
    ea = np.concatenate([c - 0.05 * u, c + 0.05 * u], axis=1)
    eb = np.concatenate([c + d0 * nrm - 0.05 * w, c + d0 * nrm + 0.05 * w], axis=1)
    p0 = np.concatenate([ea, eb], axis=1)
    mv = np.zeros_like(p0)
    mv[:, 2:] = -2e-3 * nrm
    p1 = p0 + mv + rng.normal(scale=2e-4, size=p0.shape)
    sets["near_ee"] = (p0.astype(np.float32), p1.astype(np.float32))
    off = rng.uniform(-0.02, 0.02, size=(m, 1, 2))
    tri = np.concatenate([c - 0.05 * u - 0.03 * v, c + 0.05 * u - 0.03 * v, c + 0.06 * v], axis=1)
    pnt = c + d0 * nrm + off[..., :1] * u + off[..., 1:] * v
    p0 = np.concatenate([pnt, tri], axis=1)
    mv = np.zeros_like(p0)
    mv[:, :1] = -2e-3 * nrm
    p1 = p0 + mv + rng.normal(scale=2e-4, size=p0.shape)
    sets["near_pt"] = (p0.astype(np.float32), p1.astype(np.float32))
    out = {}
    for name, (p0, p1) in sets.items():
        kinds = ("ee", "pt") if name == "random" else (name[-2:],)
        out[f"{name}_p0"], out[f"{name}_p1"] = p0, p1
        for kind in kinds:
            fn = f"{kind}_collision_time"
            t32 = np.array([ns32[fn](*(ns32["vec3"](v) for v in p0[i]), *(ns32["vec3"](v) for v in p1[i]))
                            for i in range(len(p0))], np.float32)
            t64 = np.array([ns64[fn](*(ns64["vec3"](v) for v in p0[i]), *(ns64["vec3"](v) for v in p1[i]))
                            for i in range(len(p0))], np.float64)
            out[f"{name}_t_{kind}32"], out[f"{name}_t_{kind}64"] = t32, t64
    # cubic roots of the float32 coefficients, both builds
    cr = np.load(os.path.join(HERE, "cubic_roots.npz"))
    coef = cr["coef"].astype(np.float32)
    for key, ns in (("32", ns32), ("64", ns64)):
        nr = np.zeros(len(coef), np.int32)
        roots = np.zeros((len(coef), 3), ns["scalar"])
        for i, c in enumerate(coef):
            k, r = ns["cubic_roots"](ns["vec4"](c), ns["scalar"](0.0), ns["scalar"](1.0))
            nr[i], roots[i] = k, r
        out[f"cubic_n_roots_{key}"], out[f"cubic_roots_{key}"] = nr, roots
    out["cubic_coef32"] = coef
    np.savez_compressed(os.path.join(HERE, "fp32_build.npz"), **out)


def make_narrow32(ref: str):
    """I. the narrow phase of the reference's float32 build
    (dynamic_contacts.py:152-246, 375-398 with scalar = float32) on the scene
    of narrow_fp64.npz rounded to float32."""
    d = np.load(os.path.join(HERE, "narrow_fp64.npz"))
    ns32 = reference_ns(ref, fp64=False)
    x32 = d["x"].astype(np.float32)
    xcs32 = d["xcs"].astype(np.float32)
    th = np.float32(d["l0"]) * np.float32(0.5)
    ns32["_thickness"] = float(th)
    ns32["buffer"] = float(th)
    states = types.SimpleNamespace(x=x32)
    soup = types.SimpleNamespace(edges=d["edges"], triangles=d["triangles"], body=d["body"], x_transformed=x32,
                                 xcs=xcs32)
    lists = {}
    for kind in ("ee", "pt"):
        rec = d[kind]
        c = make_contacts(ns32, max(len(rec), 1))
        for k, r in enumerate(rec):
            c.list[k] = ns32["XConstraint"](a1a2b1b2=ns32["wp"].vec4i(r[:4]), e0e1=ns32["wp"].vec2i(r[4:]),
                                            l0=np.float32(2) * th, alpha=np.float32(0), lam=np.float32(0))
        c.cnt[0] = len(rec)
        lists[kind] = c
    n_ee, n_pt = len(d["ee"]), len(d["pt"])
    kappa = np.float32(d["kappa"])
    trip = types.SimpleNamespace(rows=np.zeros(16 * (n_ee + n_pt), np.int32),
                                 cols=np.zeros(16 * (n_ee + n_pt), np.int32),
                                 vals=np.zeros((16 * (n_ee + n_pt), 3, 3), np.float32))
    b = np.zeros_like(x32)
    wp.launch(ns32["contact_hessian_ee"], n_ee, states, soup, lists["ee"].list, trip, b, kappa)
    wp.launch(ns32["contact_hessian_pt"], n_pt, states, soup, lists["pt"].list, trip, b, n_ee, kappa)
    e = np.zeros(1, np.float32)
    wp.launch(ns32["contact_energy_ee"], n_ee, states, soup, lists["ee"].list, e, kappa)
    e_ee = e[0]
    e[0] = 0
    wp.launch(ns32["contact_energy_pt"], n_pt, states, soup, lists["pt"].list, e, kappa)
    np.savez_compressed(os.path.join(HERE, "narrow_fp32.npz"), x=x32, xcs=xcs32, l0=np.float32(2) * th,
                        rows=trip.rows, cols=trip.cols, vals=trip.vals, force=b, e_ee=e_ee, e_pt=e[0])


def main(ref: str, sections=("A", "B", "C", "D", "E", "F", "G", "H", "I")):
    if "F" in sections:
        make_fem(ref)
    if "G" in sections:
        make_abd(ref)
    if "H" in sections:
        make_fp32(ref)
    if "I" in sections:
        make_narrow32(ref)
    if not set(sections) & set("ABCDE"):
        print("golden vectors written:", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
        return
    from ipc_warp_b200 import scenes

    rng = np.random.default_rng(2024)
    out = {}

    # A. closest_point_triangle (contact.py:230-302), float32
    ns32 = reference_ns(ref, fp64=False)
    P = rng.normal(size=(4000, 4, 3)).astype(np.float32)
    P[:1000, 0] = (P[:1000, 1] + 0.3 * (P[:1000, 2] - P[:1000, 1]) + 0.3 * (P[:1000, 3] - P[:1000, 1])
                   + 1e-3 * rng.normal(size=(1000, 3))).astype(np.float32)
    uvd = np.zeros((len(P), 3), np.float32)
    ty = np.zeros(len(P), np.int32)
    for i, p in enumerate(P):
        r, t = ns32["closest_point_triangle"](p[0], p[1], p[2], p[3])
        uvd[i], ty[i] = r, t
    np.savez_compressed(os.path.join(HERE, "closest_point_triangle.npz"), pts=P, uvd=uvd, type=ty)

    # B. cubic_roots (cubic_roots.py:96-193), float64, on [0, 1]
    ns64 = reference_ns(ref, fp64=True)
    np.random.seed(7)
    c3, r3 = ns64["construct_3_root_polynomial"](600, 1.0)
    cr = rng.normal(size=(600, 4))
    cq = rng.normal(size=(200, 4))
    cq[:, 3] = 0.0
    coef = np.concatenate([c3, cr, cq]).astype(np.float64)
    nroots = np.zeros(len(coef), np.int32)
    roots = np.zeros((len(coef), 3))
    for i, c in enumerate(coef):
        n, r = ns64["cubic_roots"](ns64["vec4"](c), np.float64(0.0), np.float64(1.0))
        nroots[i], roots[i] = n, r
    np.savez_compressed(os.path.join(HERE, "cubic_roots.npz"), coef=coef, n_roots=nroots, roots=roots,
                        constructed_roots=r3)

    # C. DCD candidate lists (contact.py:199-336), float32 build
    sc = scenes.two_cubes(n=3, gap=3e-4, seed=2)
    dcd = {}
    for exclude in (False, True):
        ee, pt, _, _ = run_dcd(ns32, sc, sc.x.astype(np.float32), exclude)
        dcd[f"ee_{int(exclude)}"], dcd[f"pt_{int(exclude)}"] = ee, pt
    np.savez_compressed(os.path.join(HERE, "dcd_two_cubes_3.npz"), x=sc.x.astype(np.float32), edges=sc.edges,
                        triangles=sc.triangles, body=sc.body, thickness=np.float32(sc.thickness), **dcd)

    # D. per-pair collision times (ccd.py:304-357), float64
    n = 1500
    p0 = rng.normal(size=(n, 4, 3))
    p1 = p0 + rng.normal(scale=0.7, size=(n, 4, 3))
    tee = np.array([ns64["ee_collision_time"](*(ns64["vec3"](v) for v in p0[i]), *(ns64["vec3"](v) for v in p1[i]))
                    for i in range(n)])
    tpt = np.array([ns64["pt_collision_time"](*(ns64["vec3"](v) for v in p0[i]), *(ns64["vec3"](v) for v in p1[i]))
                    for i in range(n)])
    np.savez_compressed(os.path.join(HERE, "collision_time.npz"), p0=p0, p1=p1, t_ee=tee, t_pt=tpt)

    # E. narrow phase composition (dynamic_contacts.py:152-246, 375-398), float64 build
    sc = scenes.two_cubes(n=4, gap=2e-4, angle_deg=30.0, seed=4)
    x64 = sc.x.astype(np.float64)
    x64[sc.body == 1] += np.array([0.0, -1e-4, 0.0])
    _, _, ee, pt = run_dcd(ns64, sc, x64, False)
    kappa = 1e4
    states = types.SimpleNamespace(x=x64)
    soup = types.SimpleNamespace(edges=sc.edges, triangles=sc.triangles, body=sc.body, x_transformed=x64,
                                 xcs=sc.xcs.astype(np.float64))
    n_ee, n_pt = int(ee.cnt[0]), int(pt.cnt[0])
    trip = types.SimpleNamespace(rows=np.zeros(16 * (n_ee + n_pt), np.int32),
                                 cols=np.zeros(16 * (n_ee + n_pt), np.int32),
                                 vals=np.zeros((16 * (n_ee + n_pt), 3, 3)))
    b = np.zeros_like(x64)
    wp.launch(ns64["contact_hessian_ee"], n_ee, states, soup, ee.list, trip, b, np.float64(kappa))
    wp.launch(ns64["contact_hessian_pt"], n_pt, states, soup, pt.list, trip, b, n_ee, np.float64(kappa))
    e = np.zeros(1)
    wp.launch(ns64["contact_energy_ee"], n_ee, states, soup, ee.list, e, np.float64(kappa))
    e_ee = e[0]
    e[0] = 0
    wp.launch(ns64["contact_energy_pt"], n_pt, states, soup, pt.list, e, np.float64(kappa))
    e_pt = e[0]
    np.savez_compressed(os.path.join(HERE, "narrow_fp64.npz"), x=x64, xcs=soup.xcs, edges=sc.edges,
                        triangles=sc.triangles, body=sc.body, kappa=kappa, ee=records(ee), pt=records(pt),
                        l0=np.float64(2 * np.float32(sc.thickness)), rows=trip.rows, cols=trip.cols, vals=trip.vals,
                        force=b, e_ee=e_ee, e_pt=e_pt)
    print("golden vectors written:", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the ipc_warp source tree> [sections A..I]")
    main(sys.argv[1], tuple(sys.argv[2:]) or ("A", "B", "C", "D", "E", "F", "G", "H", "I"))
