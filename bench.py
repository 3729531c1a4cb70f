"""Benchmark of the per-Newton-iteration IPC contact pipeline on B200.

One step = one Newton iteration's contact block through the public API
(ipc_warp_b200.pipeline.ContactPipeline.iteration): BVH refit, EE + PT
candidate detection, narrow phase (force + 16 Hessian triplets per record),
BSR assembly, barrier energy and the CCD step bound.

Workloads (synthetic, seeded; the reference ships none of its scene assets):

* screw_nut (the headline): a bolt and a nut of a 60-degree ISO thread,
  pitch 0.1 of the 1.0 major radius, 12 turns, about 0.5M surface triangles
  and 1.23M tets per body, radial clearance 1e-4, dhat 5e-5, the nut pushed
  onto one flank (gap 0.4 dhat) and driven at 4 rad/s over dt = 2e-3;
* rod_bundle (a second line): the rod-twist configuration's 16 rods of
  4x4x256 hex cells, 5 tets/cell (102,800 vertices) in the wound contact
  state, facing rod sides 0.5 dhat apart (dhat = 1e-3 rod width).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The reference arm times the CPU oracle's restatement of the same pipeline
(the reference itself is Warp + an empty ipctkwp submodule and cannot run).
For N > 1 every rank runs an independent replica (the reference path is a
single-GPU simulator); value = pairs processed by all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton step ms, learned-PCG vs cuDSS at rel res 1e-6; contact pairs/s, %HBM"
WORKLOADS = {
    "screw_nut": "screw_nut_iso60_pitch0.1_12turns_0.5Mtris_per_body_loaded_flank_driven_4rad_s",
    "rod_bundle": "rod_twist_16rods_4x4x256_wound_contact_state",
}
HEADLINE = "screw_nut"

ROD_SIDE = 4  # rods per side of the bundle; --rods N shrinks the workload for profiler captures
TURNS = 12  # thread turns of the screw and nut; --turns N shrinks it for profiler captures


def scene(name: str = HEADLINE):
    from ipc_warp_b200 import scenes

    if name == "screw_nut":
        return scenes.screw_and_nut(turns=TURNS)
    return scenes.rod_bundle(n_rods_side=ROD_SIDE, cells=(4, 4, 256), width=0.1, gap_over_dhat=0.5,
                             jitter_over_dhat=0.05, seed=1, kappa=1e4)


def direction(sc):
    """The workload's Newton direction (x1 = x - dx)."""
    from ipc_warp_b200 import scenes

    if sc.name.startswith("screw_nut"):
        return scenes.screw_direction(sc)
    return newton_direction(sc)


def newton_direction(sc, seed=2):
    """Seeded stand-in for a Newton step of the rod bundle: neighbours
    approach by ~dhat."""
    rng = np.random.default_rng(seed)
    dx = rng.normal(scale=0.3 * sc.dhat, size=sc.x.shape)
    width = sc.meta["width"]
    centre = sc.x.reshape(-1, 3).mean(0)
    # squeeze the bundle toward its axis (x -= dx)
    dx[:, :2] += 0.02 * (sc.x[:, :2] - centre[:2]) / width * sc.dhat
    return dx


# ------------------------------------------------------------------ timing
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        """Sample every 50 ms from before the warm-up to after the e2e loop."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [c.strip() for c in line.split(",")]
            if len(f) >= 9 and f[1].replace(".", "").isdigit():
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit()),
                "reasons": reasons}


def flush_l2(buf):
    buf.add_(1.0)  # 256 MiB write > 126 MB L2


def count_kernels(fn):
    """Number of this library's kernels one call of fn launches."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    names = [e.name for e in prof.events() if e.device_type.name == "CUDA"]
    ours = [n for n in names if "ipcb" in n]
    return len(ours), sorted(set(ours))


# ---------------------------------------------------------------- roofline
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# algorithmic bytes per pair of the narrow-phase kernel (float32 records):
# record 24 + positions 48 + 16 triplets (4+4+36) 704 + force 48; EE adds rest positions 48
NARROW_BYTES = {"pt": 824, "ee": 872}
# dram__bytes_read.sum + dram__bytes_write.sum of the EE + PT narrow-phase
# launches (k_contact_hessian_sorted) of one step: one-pass ncu capture of each
# full workload
NARROW_DRAM_BYTES_PER_STEP = {"rod_bundle": 464.2e6, "screw_nut": 169.6e6}
# DRAM bytes (read + write) of the CCD edge-edge query per step -- k_ee_collect
# (both passes), k_cand_bound, k_cand_bucket, k_cand_solve -- from one ncu pass
# of dram__bytes_read.sum + dram__bytes_write.sum on the full workload (caches
# flushed before each launch, so an upper bound on the in-step traffic)
CCD_DRAM_BYTES_PER_STEP = {"rod_bundle": 41.6e6, "screw_nut": 342.1e6}


def stage_times(pipe, dx, reps, torch):
    """Per-stage device times (ms, mean over reps) on the launching stream;
    the narrow phase is the class-sorted path the pipeline runs (its two
    ordering kernels included)."""
    from ipc_warp_b200 import _native as N
    from ipc_warp_b200.dynamic_contacts import contact_hessian_ee, contact_hessian_pt

    st = torch.cuda.current_stream()
    acc = {}

    def ev():
        e = torch.cuda.Event(enable_timing=True)
        e.record(st)
        return e

    n_ee, n_pt = pipe.n_contacts, pipe.n_contacts_pt
    t = pipe.collision_triplets
    for _ in range(reps):
        marks = [("start", ev())]
        pipe.update_bvh()
        marks.append(("refit", ev()))
        pipe._launch_dcd("ee")
        marks.append(("dcd_ee", ev()))
        pipe._launch_dcd("pt")
        marks.append(("dcd_pt", ev()))
        pipe.b.zero_()
        contact_hessian_ee(None, pipe.soup, pipe.contacts_new, t, pipe.b, pipe.contact_stiffness, n=n_ee,
                           ws=pipe._ws_ee)
        marks.append(("narrow_ee", ev()))
        contact_hessian_pt(None, pipe.soup, pipe.contacts_pt, t, pipe.b, n_ee, pipe.contact_stiffness, n=n_pt,
                           ws=pipe._ws_pt)
        marks.append(("narrow_pt", ev()))
        from ipc_warp_b200.bsr import contact_bsr

        contact_bsr(pipe.contacts_new, n_ee, pipe.contacts_pt, n_pt, pipe.soup.n_verts, t,
                    out=pipe.collision_hessian)
        marks.append(("bsr", ev()))
        pipe.compute_collision_energy(detect=False)
        marks.append(("energy", ev()))
        # the CCD of collision_free_step, stage by stage: swept boxes + refit,
        # then each query (candidate collection + candidate solve, one call)
        soup = ctypes.byref(pipe.soup.c_struct())
        s = N.stream_handle()
        N.call("ipcb_add_dx", soup, N.ptr(dx), N.ptr(pipe.ccd_x1), s)
        N.call("ipcb_swept_edge_aabbs", soup, N.ptr(pipe.ccd_x1), 1e-7, N.ptr(pipe.ccd_edge_lower),
               N.ptr(pipe.ccd_edge_upper), s)
        pipe.ccd_edge_bvh.refit(pipe.ccd_edge_lower, pipe.ccd_edge_upper)
        pipe.ccd_toi.fill_(1.0)
        pipe._status.zero_()
        marks.append(("ccd_boxes_ee", ev()))
        N.call("ipcb_edge_edge_toi", soup, N.ptr(pipe.ccd_x1), ctypes.byref(pipe.ccd_edge_bvh.c),
               N.ptr(pipe.ccd_edge_lower), N.ptr(pipe.ccd_edge_upper), int(pipe.disable_self_collision),
               N.ptr(pipe.ccd_toi), N.ptr(pipe._status), N.ptr(pipe._toi_ws), pipe._toi_ws.numel(), s)
        marks.append(("ccd_query_ee", ev()))
        N.call("ipcb_swept_triangle_aabbs", soup, N.ptr(pipe.ccd_x1), 1e-7, N.ptr(pipe.ccd_triangle_lower),
               N.ptr(pipe.ccd_triangle_upper), s)
        pipe.ccd_triangle_bvh.refit(pipe.ccd_triangle_lower, pipe.ccd_triangle_upper)
        marks.append(("ccd_boxes_pt", ev()))
        N.call("ipcb_point_triangle_toi", soup, N.ptr(pipe.ccd_x1), ctypes.byref(pipe.ccd_triangle_bvh.c), 1e-7,
               int(pipe.disable_self_collision), N.ptr(pipe.ccd_toi), N.ptr(pipe._status), N.ptr(pipe._toi_ws_pt),
               pipe._toi_ws_pt.numel(), s)
        marks.append(("ccd_query_pt", ev()))
        torch.cuda.synchronize()
        for (a, ea), (b, eb) in zip(marks[:-1], marks[1:]):
            acc[b] = acc.get(b, 0.0) + ea.elapsed_time(eb) / reps
    return acc


# ------------------------------------------------------------- Newton step
NEWTON_WORKLOAD = "rod_twist_16rods_4x4x256_wound_theta0.3_stvk_dt5e-3_kappa1e13"
NEWTON_KAPPA = 1e13


def newton_solver(dev, torch, linear_solver: str, preconditioner: str, theta: float = 0.3):
    """FEMContactSolver on the rod-twist bundle in a wound state: the
    cross-sections turned by up to +-theta, the clamped ends advancing by one
    step of the 2 rad/s counter-rotation (StVK, E = 1e6, nu = 0.45, dt = 5e-3,
    rel. residual 1e-6)."""
    from ipc_warp_b200 import scenes
    from ipc_warp_b200.newton import FEMContactSolver

    sc = scene("rod_bundle")
    # barrier stiffness scaled to dhat = 1e-4 (energies of order kappa dhat^4 = 1e-3 J);
    # the pipeline workload's kappa does not change its work, but a Newton step needs it
    sc.kappa = NEWTON_KAPPA
    fixed, at = scenes.twist_targets(sc, omega=2.0)
    s = FEMContactSolver(sc, material="stvk", E=1e6, nu=0.45, h=5e-3, fixed=fixed, gravity=(0.0, 0.0, 0.0),
                         dtype=torch.float32, device=dev, tol=1e-6, maxiter=20000, linear_solver=linear_solver,
                         preconditioner=preconditioner)
    x = torch.tensor(scenes.twist_bundle(sc, theta), dtype=torch.float32, device=dev)
    s.states.x.copy_(x)
    s.states.x0.copy_(x)
    tgt = at(0.0)
    tgt[fixed] = scenes.twist_bundle(sc, theta + 2.0 * 5e-3)[fixed]
    s.x_target.copy_(torch.tensor(tgt, dtype=torch.float32))
    return s


def newton_step_times(dev, torch, reps: int = 3, direct_reps: int = 1):
    """ms of one full Newton iteration (compute_A -> rhs -> solve -> line
    search, CUDA events around it) for learned-PCG, block-Jacobi PCG and the
    direct Cholesky solve, from the same state."""
    out = {"workload": NEWTON_WORKLOAD, "rel_res": 1e-6, "ms": {}, "phase_ms": {}, "pcg_iterations": {},
           "alpha": {}}
    for name, ls, pc in (("learned_pcg", "pcg", "learned"), ("jacobi_pcg", "pcg", "jacobi"),
                         ("direct_cholesky", "direct", "jacobi")):
        s = newton_solver(dev, torch, ls, pc)
        s.timing = True
        x0 = s.states.x.clone()
        n = direct_reps if ls == "direct" else reps
        times = []
        for r in range(n + (0 if ls == "direct" else 1)):  # one untimed warm-up for the PCG paths
            s.states.x.copy_(x0)
            s.stats.pcg_iterations.clear()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            alpha, _ = s.newton_iteration()
            b.record()
            torch.cuda.synchronize()
            if ls == "direct" or r > 0:
                times.append(a.elapsed_time(b))
        out["ms"][name] = statistics.median(times)
        out["phase_ms"][name] = {k: round(v, 3) for k, v in s.phase_ms.items()}
        out["pcg_iterations"][name] = s.stats.pcg_iterations[-1] if s.stats.pcg_iterations else None
        out["alpha"][name] = alpha
        out["n_contacts"] = s.n_contacts + s.n_contacts_pt
        del s
        torch.cuda.empty_cache()
    # one whole time step (Newton to convergence, max|dx| <= 5e-2 h as the
    # reference's default) from the same state; the learned factor is built
    # once per step and reused by the later iterations of the step
    out["time_step"] = {}
    for name, pc, refresh in (("learned_pcg_factor_per_step", "learned", 10 ** 6), ("jacobi_pcg", "jacobi", 1)):
        s = newton_solver(dev, torch, "pcg", pc)
        s.precond_refresh = refresh
        s.max_newton = 60
        x0 = s.states.x.clone()
        times = []
        for r in range(2):
            s.states.x.copy_(x0)
            s.states.x0.copy_(x0)
            s.states.xdot.zero_()
            s.time = 0.0
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            st = s.step()
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
        out["time_step"][name] = {"ms": times[-1], "newton_iterations": st.newton_iterations,
                                  "pcg_iterations": sum(st.pcg_iterations)}
        del s
        torch.cuda.empty_cache()
    ms = out["ms"]
    out["speedup_learned_vs_direct"] = ms["direct_cholesky"] / ms["learned_pcg"]
    out["speedup_learned_vs_jacobi"] = ms["jacobi_pcg"] / ms["learned_pcg"]
    solve = {k: v["solve"] for k, v in out["phase_ms"].items()}
    out["solve_speedup_learned_vs_direct"] = solve["direct_cholesky"] / solve["learned_pcg"]
    out["solve_speedup_learned_vs_jacobi"] = solve["jacobi_pcg"] / solve["learned_pcg"]
    out["direct_solver"] = "cuSOLVER csrchol with METIS ordering (cuDSS is not in this toolkit)"
    return out


WRECKING_WORKLOAD = "wrecking_balls_64_icospheres_2562v_512_nh_cubes_4x4x4_ground_100x100_dt1e-2_kappa1e12"


def wrecking_balls_steps(dev, torch, before: int = 55, timed: int = 3):
    """The batched affine + FEM wrecking balls (64 pendulum icospheres, 512
    neo-Hookean cubes, fixed ground) in one mixed Newton solve: ``before``
    untimed time steps (the balls swing into their cube stacks), then
    ``timed`` steps timed with CUDA events, the phases of one Newton
    iteration at the last state, and the intersection check."""
    from ipc_warp_b200 import scenes
    from ipc_warp_b200.mixed import MixedSolver

    sc = scenes.wrecking_balls(n_balls=64)
    s = MixedSolver(sc, E=5e5, nu=0.4, h=1e-2, dtype=torch.float32, device=dev, maxiter=2000)
    for _ in range(before):
        s.step()
    steps = []
    for _ in range(timed):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        st = s.step()
        b.record()
        torch.cuda.synchronize()
        steps.append({"ms": a.elapsed_time(b), "newton_iterations": st.newton_iterations,
                      "pcg_iterations": st.pcg_iterations, "records": s.n_contacts + s.n_contacts_pt})
    s.prepare()
    phase = {}
    for name, fn in (("compute_A", s.compute_A), ("solve", s.solve), ("line_search", s.line_search)):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        phase[name] = round(a.elapsed_time(b), 3)
    key = next(iter(s._tuner.best.values()), None) if s._tuner.best else None
    return {"workload": WRECKING_WORKLOAD, "unknowns": s.nq, "vertices": s.n_verts, "tets": s.n_tets,
            "bodies": s.n_bodies, "steps_before": before, "timed_steps": steps,
            "ms_per_step": statistics.median(x["ms"] for x in steps), "newton_iteration_phase_ms": phase,
            "terms_schedules": {k: list(v) for k, v in s._tuner.best.items()}, "last_schedule": key,
            "edge_triangle_crossings": s.edge_triangle_crossings()[0],
            "orthogonality_error": s.orthogonality_error()}


def run_profile_mixed():
    """One Newton iteration of the wrecking balls at an impact state (after
    55 steps), between cudaProfilerStart/Stop (ncu --profile-from-start off)."""
    import torch

    from ipc_warp_b200 import scenes
    from ipc_warp_b200.mixed import MixedSolver

    dev = torch.device("cuda", 0)
    s = MixedSolver(scenes.wrecking_balls(n_balls=64), E=5e5, nu=0.4, h=1e-2, dtype=torch.float32, device=dev,
                    maxiter=2000)
    for _ in range(55):
        s.step()
    s.prepare()
    s.newton_iteration()  # buffers and graphs at this state
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    s.newton_iteration()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()


def run_profile_solver(args):
    """Untimed launches of the Newton solve's kernels on the wound rod bundle
    (for ncu): two learned-factor builds (MPNN forward, row normalisation,
    bf16 mirror) and two short PCG solves (learned factor, block Jacobi)."""
    import torch

    from ipc_warp_b200 import learned as L
    from ipc_warp_b200.newton import DevicePcg, JacobiPrecond

    dev = torch.device("cuda", 0)
    s = newton_solver(dev, torch, "pcg", "jacobi")
    s.compute_A()
    s.compute_rhs()
    net = L.Net.load(L.DEFAULT_WEIGHTS, device=dev)
    for _ in range(2):
        M = L.LearnedFactor(net, s.A)
    dp = DevicePcg(batch=4, use_graph=False)
    dp.solve(s.A, s.rhs, M, 1e-6, 8)
    dp.solve(s.A, s.rhs, JacobiPrecond(s.A), 1e-6, 8)
    torch.cuda.synchronize()


def run_profile_newton(args):
    """Untimed Newton iterations on the wound rod bundle (for ncu launch
    lists): one warm-up iteration, then two more between
    cudaProfilerStart/Stop, each compute_A (work-queue terms + fixed-pattern
    assembly), rhs, learned-PCG solve, device line search."""
    import torch

    dev = torch.device("cuda", 0)
    s = newton_solver(dev, torch, "pcg", "learned")
    x0 = s.states.x.clone()
    s.newton_iteration()  # warm-up: autotuning, graph captures, buffer pools
    torch.cuda.synchronize()
    torch.cuda.profiler.start()  # ncu --profile-from-start off captures from here
    for _ in range(2):
        s.states.x.copy_(x0)
        s.newton_iteration()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()


# ------------------------------------------------------------- CPU oracle
def cpu_pipeline(sc, dx, reps):
    """One pass of the oracle's restatement: DCD EE + PT, narrow phase
    (analytic subspace route: force, Hessian, energy), contact BSR assembly,
    scene TOI.  Returns (pairs, seconds/pass)."""
    from oracle import pyoracle as po

    x32 = sc.x.astype(np.float32)
    x1 = x32 - dx.astype(np.float32)
    th = np.float32(sc.thickness)
    times = []
    pairs = 0
    for _ in range(reps):
        t0 = time.perf_counter()
        ee = po.dcd_ee(x32, sc.edges, sc.body, th, cap=1 << 21)
        pt = po.dcd_pt(x32, sc.triangles, sc.body, th, cap=1 << 21)
        l0e = np.full(len(ee), th * np.float32(2), np.float32)
        l0p = np.full(len(pt), th * np.float32(2), np.float32)
        _, He, _, _ = po.narrow("ee", ee[:, :4], l0e, x32, sc.xcs.astype(np.float32), sc.kappa, mode=1)
        _, Hp, _, _ = po.narrow("pt", pt[:, :4], l0p, x32, None, sc.kappa, mode=1)
        po.contact_bsr(sc.n_verts, np.concatenate([ee[:, :4], pt[:, :4]]), np.concatenate([He, Hp]))
        del He, Hp
        po.scene_toi(x32, x1, sc.edges, sc.triangles, sc.body)
        times.append(time.perf_counter() - t0)
        pairs = len(ee) + len(pt)
    return pairs, statistics.mean(times)


def run_reference(args):
    """CPU arm: the oracle pipeline on all host threads, K timed passes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc = scene(args.workload)
    dx = direction(sc)
    cores = os.cpu_count()
    cpu_pipeline(sc, dx, max(args.warmup, 1))
    pairs, sec = cpu_pipeline(sc, dx, args.steps)
    value = pairs / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.workload, sc, pairs),
        "details": {"parallelism": f"{cores} host threads (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "port",
                         "sample": "full workload, one DCD+narrow+energy+BSR+CCD pass per step (C++ oracle, OpenMP)"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


L2_NOTE = "GPU arm: L2 flushed between timed steps (256 MiB write)"


def workload_config(name, sc, pairs):
    """The config both arms report for a workload (identical keys and values;
    run details go beside it, in ``details``)."""
    return {"workload": WORKLOADS[name], "verts": sc.n_verts, "edges": sc.n_edges, "tris": sc.n_tris,
            "dhat": sc.dhat, "pairs": pairs, "l2": L2_NOTE}


def max_over_ranks(values, device):
    """Per-rank device timings (ms) -> their maxima over the process group
    (the slowest replica sets the whole job's time)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def job_throughput(world: int, pairs: int, steps: int, total_ms: float) -> float:
    """Whole-job pairs/s of N replicas that each processed `pairs` per step."""
    return world * pairs * steps / (total_ms * 1e-3)


def measure(name, args, dev, world, rank, torch, dist, full: bool):
    """Time one workload: K device-timed steps (L2 flushed between steps),
    then K end-to-end steps with host positions and direction copied in and
    the force copied out.  With ``full`` (rank 0), also the stage times, the
    roofline of the narrow phase, the CPU baseline and the kernel count."""
    from ipc_warp_b200.pipeline import ContactPipeline

    sc = scene(name)
    dx_np = direction(sc)
    pipe = ContactPipeline.from_scene(sc, dtype=torch.float32, device=dev)
    dx = torch.tensor(dx_np, dtype=torch.float32, device=dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def step():
        return pipe.iteration(dx)

    for _ in range(max(args.warmup, 3)):
        r = step()
    torch.cuda.synchronize()
    pairs = r.n_ee + r.n_pt
    if args.profile_only:
        torch.cuda.profiler.start()  # ncu --profile-from-start off captures the K steps only
        for _ in range(args.steps):
            step()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        return None

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    evs = []
    for _ in range(args.steps):
        flush_l2(flush)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        step()
        e.record()
        evs.append((s, e))
    barrier()
    total_ms = sum(s.elapsed_time(e) for s, e in evs)

    # ---- end to end: pinned host inputs copied in, results read back
    xh = torch.tensor(sc.x, dtype=torch.float32).pin_memory()
    dxh = dx.cpu().pin_memory()
    bh = torch.empty_like(pipe.b, device="cpu").pin_memory()
    # the host-buffer call: x and dx copied in, the force copied out, the
    # copies inside the replayed sequence (dx and b overlap other stages)
    pipe.iteration_host(xh, dxh, bh)
    e2e_ev = []
    barrier()
    for _ in range(args.steps):
        flush_l2(flush)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        pipe.iteration_host(xh, dxh, bh)
        e.record()
        e2e_ev.append((s, e))
    barrier()
    e2e_ms = sum(s.elapsed_time(e) for s, e in e2e_ev)
    h2d = xh.numel() * 4 + dxh.numel() * 4
    d2h = bh.numel() * 4 + 8 + 4 + 16  # force, energy, toi, counts + statuses
    if world > 1:
        total_ms, e2e_ms = max_over_ranks([total_ms, e2e_ms], dev)
    out = {"workload": WORKLOADS[name], "pairs": pairs, "n_ee": r.n_ee, "n_pt": r.n_pt,
           "value": job_throughput(world, pairs, args.steps, total_ms), "ms_per_step": total_ms / args.steps,
           "e2e": {"value": job_throughput(world, pairs, args.steps, e2e_ms), "unit": "pairs/s",
                   "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
           "sc": sc}
    if not full:
        return out
    st = stage_times(pipe, dx, 5, torch)
    ws = [int(v) for v in torch.cat([pipe._toi_ws[:4].view(torch.int32), pipe._toi_ws_pt[:4].view(torch.int32)])]
    n_launch, names = count_kernels(step)
    peak, peak_kind = peaks()
    n_ee, n_pt = pipe.n_contacts, pipe.n_contacts_pt
    narrow_ms = st["narrow_ee"] + st["narrow_pt"]
    algo = n_ee * NARROW_BYTES["ee"] + n_pt * NARROW_BYTES["pt"]
    achieved = algo / (narrow_ms * 1e-3) / 1e9
    narrow_roof = {"kernel": "k_contact_hessian_sorted (EE + PT, with its two ordering kernels)", "bound": "hbm",
                   "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                   "frac": achieved / peak, "traffic": NARROW_DRAM_BYTES_PER_STEP[name], "algorithmic_bytes": algo}
    # CCD edge-edge query: 56 B per query edge (its box and ids) + 112 B per
    # staged candidate (pair, 8 positions at t0 and t1), per the survey's
    # per-unit figures; it is the largest stage on the screw and nut
    ccd_algo = 56 * pipe.soup.n_edges + 112 * ws[0]
    ccd_achieved = ccd_algo / (st["ccd_query_ee"] * 1e-3) / 1e9
    ccd_roof = {"kernel": "k_ee_collect + k_cand_toi (CCD edge-edge query)", "bound": "hbm",
                "achieved": ccd_achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": ccd_achieved / peak, "traffic": CCD_DRAM_BYTES_PER_STEP[name], "algorithmic_bytes": ccd_algo,
                "note": "bound by the double-precision root isolation and the dependent position gathers, "
                        "not by DRAM"}
    dominant = "ccd" if st["ccd_query_ee"] > narrow_ms else "narrow"
    cpu_pairs, cpu_sec = cpu_pipeline(sc, dx_np, 3)
    out.update({
        "ccd_candidates": ws[0] + ws[1],
        "stage_ms": {k: round(v, 4) for k, v in st.items()},
        "roofline": ccd_roof if dominant == "ccd" else narrow_roof,
        "roofline_narrow": narrow_roof,
        "roofline_ccd": ccd_roof,
        "cpu_baseline": {"value": cpu_pairs / cpu_sec, "unit": "pairs/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": "full workload, 3 passes of the C++ oracle pipeline (DCD+narrow+energy+BSR+CCD)"},
        "gpu_launches": n_launch * args.steps, "kernels": names,
    })
    return out


def run_sharded(args):
    """``--shard``: one scene split over the N ranks (ipc_warp_b200.sharded:
    query ranges, force / energy / TOI exchanged over NCCL); K device-timed
    steps after W warm-up steps, max over ranks; value = the scene's pairs
    per second (strong scaling)."""
    import torch
    import torch.distributed as dist

    from ipc_warp_b200.sharded import ShardedContactPipeline

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    sc = scene(args.workload)
    dx = torch.tensor(direction(sc), dtype=torch.float32, device=dev)
    pipe = ShardedContactPipeline.from_scene(sc, rank, world, dtype=torch.float32, device=dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(max(args.warmup, 3)):
        r = pipe.iteration(dx)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    evs = []
    for _ in range(args.steps):
        flush_l2(flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        r = pipe.iteration(dx)
        b.record()
        evs.append((a, b))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    total = sum(a.elapsed_time(b) for a, b in evs)
    if world > 1:
        total, _ = max_over_ranks([total, total], dev)
    pairs = r.n_ee_total + r.n_pt_total
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": pairs * args.steps / (total * 1e-3), "unit": "pairs/s",
                          "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
                          "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": workload_config(args.workload, sc, pairs),
                          "details": {"parallelism": f"sharded x{world}"}}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    sampler = ClockSampler(local)
    if not args.profile_only:
        sampler.start()
    head = measure(args.workload, args, dev, world, rank, torch, dist, full=rank == 0)
    if args.profile_only:
        return
    second = None
    if not args.headline_only:
        other = "rod_bundle" if args.workload != "rod_bundle" else "screw_nut"
        second = measure(other, args, dev, world, rank, torch, dist, full=rank == 0)
    clocks = sampler.stop()
    out = None
    if rank == 0:
        newton = None if args.no_newton else newton_step_times(dev, torch)
        wrecking = None if args.no_newton else wrecking_balls_steps(dev, torch)
        sc = head.pop("sc")
        cfg = workload_config(args.workload, sc, head["pairs"])
        details = {"n_ee": head["n_ee"], "n_pt": head["n_pt"], "ccd_candidates": head["ccd_candidates"],
                   "parallelism": f"replicas x{world}", "stage_ms": head["stage_ms"]}
        out = {
            "metric": METRIC, "value": head["value"], "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg, "details": details, "roofline": head["roofline"],
            "roofline_narrow": head["roofline_narrow"], "roofline_ccd": head["roofline_ccd"],
            "cpu_baseline": head["cpu_baseline"],
            "e2e": head["e2e"], "gpu_launches": head["gpu_launches"], "kernels": head["kernels"], "clocks": clocks,
            "newton_step": newton, "wrecking_balls": wrecking,
        }
        if second is not None:
            second.pop("sc")
            second.pop("kernels", None)
            out["second_workload"] = second
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile-only", action="store_true",
                    help="warmup + K steps only (for ncu launch lists); prints nothing")
    ap.add_argument("--no-newton", action="store_true",
                    help="skip the Newton-step timing (learned-PCG / Jacobi-PCG / direct) and the wrecking balls")
    ap.add_argument("--profile-solver", action="store_true",
                    help="untimed Newton-solve kernels only (learned factor + PCG), for ncu; prints nothing")
    ap.add_argument("--workload", default=HEADLINE, choices=sorted(WORKLOADS),
                    help="headline workload (the other one is measured as a second line)")
    ap.add_argument("--headline-only", action="store_true", help="skip the second workload")
    ap.add_argument("--turns", type=int, default=12,
                    help="thread turns of the screw and nut (12 = the benchmark workload; fewer for ncu captures)")
    ap.add_argument("--rods", type=int, default=4,
                    help="rods per side of the bundle (4 = the benchmark workload; smaller for ncu section captures)")
    ap.add_argument("--shard", action="store_true",
                    help="split the headline workload over the N ranks (strong scaling) instead of N replicas")
    ap.add_argument("--profile-newton", action="store_true",
                    help="untimed Newton iterations (learned PCG, device line search), for ncu; prints nothing")
    ap.add_argument("--profile-mixed", action="store_true",
                    help="wrecking balls: 55 untimed steps, then one Newton iteration between "
                         "cudaProfilerStart/Stop, for ncu; prints nothing")
    args = ap.parse_args()
    global ROD_SIDE, TURNS
    ROD_SIDE = args.rods
    TURNS = args.turns
    if args.profile_mixed:
        run_profile_mixed()
        return
    if args.profile_solver:
        run_profile_solver(args)
        return
    if args.profile_newton:
        run_profile_newton(args)
        return
    if args.impl == "reference":
        run_reference(args)
    elif args.shard:
        run_sharded(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
