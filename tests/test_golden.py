"""The oracle against golden vectors produced by running the reference's own
functions (tests/golden/make_golden.py).  CPU only."""
import os

import numpy as np
import pytest

from helpers import rel_err, sort_records
from oracle import pyoracle as po

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(G, name))


def test_closest_point_triangle_bit_exact():
    d = load("closest_point_triangle.npz")
    P = d["pts"]
    uvd, ty = po.closest_point_triangle(P[:, 0], P[:, 1], P[:, 2], P[:, 3])
    assert np.array_equal(ty, d["type"])
    assert np.array_equal(uvd, d["uvd"])


def test_cubic_roots_bit_exact():
    d = load("cubic_roots.npz")
    nr, roots, st = po.cubic_roots(d["coef"], 0.0, 1.0)
    assert st == 0
    assert np.array_equal(nr, d["n_roots"])
    for i in range(len(nr)):
        assert np.array_equal(roots[i, :nr[i]], d["roots"][i, :nr[i]]), i


def test_collision_time_bit_exact():
    d = load("collision_time.npz")
    assert np.array_equal(po.collision_time("ee", d["p0"], d["p1"]), d["t_ee"])
    assert np.array_equal(po.collision_time("pt", d["p0"], d["p1"]), d["t_pt"])
    assert (d["t_ee"] < 1).sum() > 20 and (d["t_pt"] < 1).sum() > 20


@pytest.mark.parametrize("exclude", [0, 1])
def test_dcd_candidates_match_reference(exclude):
    d = load("dcd_two_cubes_3.npz")
    ee = po.dcd_ee(d["x"], d["edges"], d["body"], d["thickness"], bool(exclude))
    pt = po.dcd_pt(d["x"], d["triangles"], d["body"], d["thickness"], bool(exclude))
    assert len(d[f"ee_{exclude}"]) > 0 and len(d[f"pt_{exclude}"]) > 0
    assert np.array_equal(sort_records(ee), sort_records(d[f"ee_{exclude}"]))
    assert np.array_equal(sort_records(pt), sort_records(d[f"pt_{exclude}"]))


@pytest.mark.parametrize("mode", [0, 1])
def test_narrow_phase_matches_reference_composition(mode):
    """Per-record Hessian blocks, the accumulated force and the energies in
    the double build (tolerance 1e-10 relative, per record / overall)."""
    d = load("narrow_fp64.npz")
    x, xcs, kappa, l0 = d["x"], d["xcs"], float(d["kappa"]), float(d["l0"])
    force = np.zeros_like(x)
    off = 0
    for kind, rec, e_ref in (("ee", d["ee"], d["e_ee"]), ("pt", d["pt"], d["e_pt"])):
        n = len(rec)
        F, H, E, act = po.narrow(kind, rec[:, :4], np.full(n, l0), x, xcs, kappa, fp64=True, mode=mode)
        for p in range(n):
            blk = d["vals"][(off + p) * 16:(off + p + 1) * 16]
            Href = np.zeros((12, 12))
            for ii in range(4):
                for jj in range(4):
                    Href[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3] = blk[ii * 4 + jj]
            if not act[p]:
                assert not np.any(Href)
                continue
            assert rel_err(H[p], Href) < 1e-10, (kind, p)
            for k in range(4):
                force[rec[p, k]] += F[p, 3 * k:3 * k + 3]
        assert abs(E.sum() - e_ref) <= 1e-10 * abs(e_ref)
        off += n
    assert rel_err(force, d["force"]) < 1e-10


MATERIALS = (("snh", 0), ("neo_hookean", 1), ("stvk", 2))


@pytest.mark.parametrize("material,code", MATERIALS)
@pytest.mark.parametrize("build", [64, 32])
def test_fem_matches_reference_kernels(material, code, build):
    """fem/fem.py compute_Dm + tet_kernel_sparse and compute_Psi, run by the
    reference for each material file: the oracle's blocks, forces and energy
    in double within 1e-12 of the double build, and within 2e-6 of the float32
    build (evaluated on the float32-rounded positions)."""
    d = load("fem_tets.npz")
    x, xcs, tets = d["x"], d["xcs"], d["tets"]
    if build == 32:
        x, xcs = x.astype(np.float32).astype(np.float64), xcs.astype(np.float32).astype(np.float64)
    force, blocks, energy = po.tet(code, x, xcs, tets, float(d["mu"]), float(d["lam"]))
    k = f"{material}_{build}"
    n = len(tets)
    assert np.array_equal(d[k + "_rows"].reshape(n, 4, 4), np.repeat(tets[:, :, None], 4, axis=2))
    assert np.array_equal(d[k + "_cols"].reshape(n, 4, 4), np.repeat(tets[:, None, :], 4, axis=1))
    tol = 1e-12 if build == 64 else 2e-6
    vals = d[k + "_vals"].astype(np.float64).reshape(n, 16, 3, 3)
    assert rel_err(blocks, vals) <= tol
    assert rel_err(force, d[k + "_force"]) <= tol
    assert abs(energy - d[k + "_psi"].astype(np.float64).sum()) <= tol * abs(energy)


@pytest.mark.parametrize("build", ["64", "32"])
def test_abd_matches_reference_kernels(build):
    """affine_body_dynamics.py _assemble_body_system, _body_energy,
    _reduce_contact_force and _reduce_contact_hessian run by the reference:
    oracle/abd.py within 1e-12 of the double build and 5e-6 of the float32
    build (the float32 gradient M (q - q~) loses digits to cancellation)."""
    from oracle import abd as oa

    a = load("abd_bodies.npz")
    tol = 1e-12 if build == "64" else 5e-6
    blocks, grad = oa.body_system(a["q"], a["qt"], a["M"], a["volume"], a["stiffness"], a["fixed"], float(a["h2"]))
    nb = len(a["volume"])
    rows = np.array([[4 * b + i for i in range(4) for _ in range(4)] for b in range(nb)]).ravel()
    cols = np.array([[4 * b + j for _ in range(4) for j in range(4)] for b in range(nb)]).ravel()
    assert np.array_equal(a["rows_" + build], rows) and np.array_equal(a["cols_" + build], cols)
    assert rel_err(blocks.reshape(-1, 3, 3), a["vals_" + build]) <= tol
    assert rel_err(grad.reshape(-1, 3), a["grad_" + build]) <= tol
    inertia, ortho = oa.body_energy(a["q"], a["qt"], a["M"], a["volume"], a["stiffness"], a["fixed"], float(a["h2"]))
    assert abs(inertia - a["inertia_" + build]) <= tol * abs(inertia)
    assert abs(ortho - a["ortho_" + build]) <= tol * abs(ortho)
    red = oa.reduce_force(a["f_vert"], a["rest"], a["body"], a["fixed"], nb)
    assert rel_err(red.reshape(-1, 3), a["reduced_force_" + build]) <= tol
    R, C, V = oa.reduce_hessian(a["src_rows"], a["src_cols"], a["src_vals"], a["rest"], a["body"], a["fixed"],
                                float(a["scale"]))
    assert np.array_equal(R, a["dst_rows_" + build]) and np.array_equal(C, a["dst_cols_" + build])
    assert rel_err(V, a["dst_vals_" + build]) <= tol


def test_ccd_float32_build():
    """The reference's float32 build (USE_FLOAT32, scalar_types.py:6) on the
    CCD path, run at fixture time beside its float64 build on the same
    float32 inputs (tests/golden/fp32_build.npz).

    * The oracle's double evaluation -- the arithmetic of the float32
      build here -- equals the float64 build bit for bit: per-pair times
      (ccd.py:304-357) and cubic roots (cubic_roots.py:96-193).
    * Well-conditioned motions (random, unit-scale): the float32 build's
      times are within 5e-6 of them and it finds the same impacts.
    * Near-contact motions (unit-scale primitives up to 1e-3 apart closing
      by 2e-3): the float32 build loses digits to the cancellation in the
      coplanarity cubic.  It misses impacts that the double evaluation finds,
      never the other way round, and its times scatter by about 1e-3 on both
      sides.  So the double evaluation cannot stay under the float32 times,
      and no accurate method could: the bound is held against the float64
      build instead (exactly), and the float32 build's error is stated here.
    """
    d = load("fp32_build.npz")
    for name, kinds in (("random", ("ee", "pt")), ("near_ee", ("ee",)), ("near_pt", ("pt",))):
        p0, p1 = d[name + "_p0"].astype(np.float64), d[name + "_p1"].astype(np.float64)
        for kind in kinds:
            t = po.collision_time(kind, p0, p1)
            t32 = d[f"{name}_t_{kind}32"].astype(np.float64)
            assert np.array_equal(t, d[f"{name}_t_{kind}64"]), (name, kind)
            hit, hit32 = t < 1, t32 < 1
            assert not np.any(hit32 & ~hit), (name, kind)  # the float32 build finds nothing the double misses
            if name == "random":
                assert np.array_equal(hit, hit32)
                assert np.abs(t - t32).max() <= 5e-6
            else:
                assert hit.sum() >= 0.99 * len(t)
                both = hit & hit32
                # the float32 build's scatter on near-contact motions
                assert 1e-4 < np.median(np.abs(t - t32)[both]) < 1e-2
    nr, roots, st = po.cubic_roots(d["cubic_coef32"].astype(np.float64), 0.0, 1.0)
    assert st == 0 and np.array_equal(nr, d["cubic_n_roots_64"])
    for i in range(len(nr)):
        assert np.array_equal(roots[i, :nr[i]], d["cubic_roots_64"][i, :nr[i]])


def test_narrow_phase_matches_reference_float32_build():
    """contact_hessian_ee/pt and contact_energy_ee/pt of the reference's
    float32 build on the narrow_fp64.npz scene rounded to float32
    (narrow_fp32.npz): the oracle's float mode (float32 gate and features,
    geometry and barrier in double) within 1e-5 per record, in the force
    and in the energies -- the float32 parity tolerance of this library."""
    d = load("narrow_fp32.npz")
    d64 = load("narrow_fp64.npz")
    x, xcs, l0, kappa = d["x"], d["xcs"], d["l0"], float(d64["kappa"])
    force = np.zeros(x.shape)
    off = 0
    for kind, rec, e_ref in (("ee", d64["ee"], d["e_ee"]), ("pt", d64["pt"], d["e_pt"])):
        n = len(rec)
        F, H, E, act = po.narrow(kind, rec[:, :4], np.full(n, l0, np.float32), x, xcs, kappa, fp64=False, mode=0)
        for p in range(n):
            Href = d["vals"][(off + p) * 16:(off + p + 1) * 16].astype(np.float64)
            Href = Href.reshape(4, 4, 3, 3).transpose(0, 2, 1, 3).reshape(12, 12)
            if not act[p]:
                assert not np.any(Href)
                continue
            assert rel_err(H[p], Href) < 1e-5, (kind, p)
            for k in range(4):
                force[rec[p, k]] += F[p, 3 * k:3 * k + 3]
        assert abs(E.sum() - float(e_ref)) <= 1e-5 * abs(float(e_ref))
        off += n
    assert rel_err(force, d["force"]) < 1e-5
