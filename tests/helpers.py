"""Shared test helpers: scenes, oracle/GPU comparison utilities."""
from __future__ import annotations

import numpy as np

from ipc_warp_b200 import scenes


def small_scenes():
    """Seeded scenes with contacts at a fraction of dhat (sizes the oracle
    finishes in well under a second)."""
    out = []
    out.append(scenes.two_cubes(n=8, gap=5e-4, seed=0))
    out.append(scenes.two_cubes(n=6, gap=2e-4, angle_deg=40.0, seed=3))
    out.append(scenes.rod_bundle(n_rods_side=2, cells=(2, 2, 32), width=0.1, gap_over_dhat=0.5, seed=5))
    out.append(scenes.rod_bundle(n_rods_side=3, cells=(3, 3, 24), width=0.1, gap_over_dhat=0.3,
                                 jitter_over_dhat=0.2, seed=7))
    return out


def sort_records(r):
    r = np.asarray(r, dtype=np.int64).reshape(-1, 6)
    if r.shape[0] == 0:
        return r
    order = np.lexsort(r.T[::-1])
    return r[order]


def blocks_to_dense(rows, cols, vals, ids):
    """16 triplet blocks of one record -> (12, 12) in record-slot order."""
    H = np.zeros((12, 12))
    for ii in range(4):
        for jj in range(4):
            H[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3] = vals[ii * 4 + jj]
    return H


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(b).max() if b.size else 0.0
    if den == 0.0:
        return float(np.abs(a).max()) if a.size else 0.0
    return float(np.abs(a - b).max() / den)
