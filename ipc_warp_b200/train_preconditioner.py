"""Train the learned FSAI preconditioner on Newton systems the simulator
produces, and write its weights.

    python -m ipc_warp_b200.train_preconditioner --out weights.npy

Systems come from scenes run with ``newton.FEMContactSolver``: two
neo-Hookean cubes, the upper one falling onto the lower one (the two-cube
contact setup), a bundle of StVK rods whose clamped ends counter-rotate so
that the rods wind together (the rod-twist setup, at a reduced rod
length), and packed, wound bundles at barrier stiffnesses up to 1e13 (the
contact-dominated systems of the wound bench state).  Every Newton matrix of every step is captured (a copy of the BSR),
and Adam minimises the mean Kaporin loss over random mini-batches.
"""
from __future__ import annotations

import argparse
import time

import numpy as np
import torch

from . import learned as L
from .bsr import BsrMatrix
from .newton import FEMContactSolver
from .scenes import rod_bundle, twist_targets, two_cubes


def _copy(A: BsrMatrix) -> BsrMatrix:
    nnz = A.nnz_sync()
    B = BsrMatrix(A.nrow, A.ncol, nnz, A.dtype, A.device)
    B.offsets.copy_(A.offsets)
    B.columns[:nnz].copy_(A.columns[:nnz])
    B.values[:nnz].copy_(A.values[:nnz])
    B.nnz_dev.copy_(A.nnz_dev)
    return B


def capture(solver: FEMContactSolver, steps: int, out: list, limit: int):
    """Run `steps` time steps, appending a copy of every Newton matrix."""
    orig = solver.solve

    def solve():
        if len(out) < limit:
            out.append(_copy(solver.A))
        return orig()

    solver.solve = solve
    try:
        for _ in range(steps):
            solver.step()
    finally:
        solver.solve = orig


def cube_systems(steps: int, seed: int, limit: int, dtype=torch.float32, n: int = 8):
    sc = two_cubes(n=n, gap=1e-3, angle_deg=15.0, jitter=1e-5, seed=seed, dhat=1e-3, kappa=1e4)
    fixed = sc.xcs[:, 1] <= sc.xcs[:, 1].min() + 1e-9
    s = FEMContactSolver(sc, material="neo_hookean", E=1e5, nu=0.4, h=1e-2, fixed=fixed, dtype=dtype, max_newton=20)
    out = []
    capture(s, steps, out, limit)
    return out


def rod_systems(steps: int, seed: int, limit: int, dtype=torch.float32, side: int = 2, cells=(4, 4, 64),
                gap_over_dhat: float | None = None):
    """Twisting rods; with ``gap_over_dhat`` the bundle starts packed with
    every facing pair of rod sides inside the barrier (contact-heavy
    systems)."""
    sc = rod_bundle(n_rods_side=side, cells=cells, seed=seed, kappa=1e4, gap_over_dhat=gap_over_dhat)
    fixed, at = twist_targets(sc, omega=2.0)
    s = FEMContactSolver(sc, material="stvk", E=1e6, nu=0.45, h=5e-3, fixed=fixed, gravity=(0.0, 0.0, 0.0),
                         dtype=dtype, max_newton=20)
    s.boundary = at
    out = []
    capture(s, steps, out, limit)
    return out


def wound_rod_systems(kappa: float, thetas, limit: int, dtype=torch.float32, side: int = 2, cells=(4, 4, 64),
                      steps: int = 1, seed: int = 3):
    """Rod-twist bundles packed and wound by each of ``thetas`` (the
    cross-sections turned by up to +-theta, the clamped ends one step of
    the 2 rad/s counter-rotation further), at barrier stiffness ``kappa``
    (dhat = 1e-3 rod width; kappa 1e13 is the stiffness whose energy scale
    kappa dhat^4 matches the rods' elastic energy): the contact-dominated
    systems of the bench's Newton state at a reduced size."""
    from .scenes import twist_bundle

    out = []
    for k, theta in enumerate(thetas):
        sc = rod_bundle(n_rods_side=side, cells=cells, seed=seed + k, kappa=kappa, gap_over_dhat=0.5)
        fixed, at = twist_targets(sc, omega=2.0)
        s = FEMContactSolver(sc, material="stvk", E=1e6, nu=0.45, h=5e-3, fixed=fixed, gravity=(0.0, 0.0, 0.0),
                             dtype=dtype, max_newton=10, tol=1e-6, maxiter=20000, direct_fallback=False)
        x = torch.tensor(twist_bundle(sc, theta), dtype=dtype, device=s.device)
        s.states.x.copy_(x)
        s.states.x0.copy_(x)
        tgt = at(0.0)
        tgt[fixed] = twist_bundle(sc, theta + 2.0 * 5e-3)[fixed]
        s.x_target.copy_(torch.tensor(tgt, dtype=dtype))
        capture(s, steps, out, limit)
    return out


def train(systems, steps: int = 400, batch: int = 4, lr: float = 2e-3, seed: int = 0, log_every: int = 50,
          net: L.Net | None = None, clip: float = 1.0):
    prepared = [L.System.from_bsr(A) for A in systems]
    net = net or L.Net(seed=seed, device=systems[0].device)
    tr = L.Trainer(net, lr=lr, clip=clip)
    rng = np.random.default_rng(seed)
    history = []
    for it in range(steps):
        idx = rng.choice(len(prepared), size=min(batch, len(prepared)), replace=False)
        loss = tr.step([prepared[i] for i in idx])
        history.append(loss)
        if log_every and (it % log_every == 0 or it == steps - 1):
            print(f"step {it:5d}  fsai loss {loss:+.5f}  skipped {tr.skipped}", flush=True)
    return net, history


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=L.DEFAULT_WEIGHTS)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--cube-steps", type=int, default=10)
    ap.add_argument("--rod-steps", type=int, default=12)
    ap.add_argument("--limit", type=int, default=120)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--stiff-kappas", default="1e9,1e11,1e13",
                    help="barrier stiffnesses of the wound-bundle systems (comma separated; empty: none)")
    ap.add_argument("--stiff-limit", type=int, default=60, help="systems per stiffness")
    ap.add_argument("--stiff-thetas", default="0.1,0.2,0.3", help="wind angles of the stiff bundles")
    ap.add_argument("--stiff-side", type=int, default=2, help="rods per side of the stiff bundles")
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--clip", type=float, default=1.0, help="gradient-norm clip (0: none)")
    args = ap.parse_args()
    t0 = time.time()
    systems = (cube_systems(args.cube_steps, args.seed, args.limit)
               + rod_systems(args.rod_steps, args.seed + 1, args.limit)
               + rod_systems(args.rod_steps, args.seed + 2, args.limit, side=3, cells=(4, 4, 32), gap_over_dhat=0.5))
    for kappa in [float(v) for v in args.stiff_kappas.split(",") if v]:
        thetas = tuple(float(v) for v in args.stiff_thetas.split(","))
        systems += wound_rod_systems(kappa, thetas, args.stiff_limit, steps=2, side=args.stiff_side)
    print(f"captured {len(systems)} Newton systems in {time.time() - t0:.1f} s", flush=True)
    t0 = time.time()
    net, hist = train(systems, steps=args.steps, seed=args.seed, lr=args.lr, clip=args.clip)
    torch.cuda.synchronize()
    print(f"trained {args.steps} steps in {time.time() - t0:.1f} s; final loss {np.mean(hist[-20:]):+.5f}")
    import os

    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    net.save(args.out)
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
