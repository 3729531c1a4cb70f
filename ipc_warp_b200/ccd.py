"""Cubic-root CCD surface of ccd/ccd.py and ccd/cubic_roots.py.

Batched evaluators (``ee_collision_time``, ``pt_collision_time``,
``cubic_roots``) run the device functions the TOI kernels use on explicit
inputs; the scene-level queries are ``ContactSolverBase.collision_free_step``.
All root arithmetic is double precision.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N


def _dev(a, device="cuda"):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device)


def collision_time(kind: str, p_t0, p_t1, device="cuda"):
    """Per-pair TOI (ccd.py:304-357).  p_t0, p_t1: (n, 4, 3); EE order
    (ei0, ei1, ej0, ej1), PT order (p, t0, t1, t2).  Returns (t, status)."""
    a, b = _dev(p_t0, device).reshape(-1, 12), _dev(p_t1, device).reshape(-1, 12)
    n = a.shape[0]
    t = torch.zeros(n, dtype=torch.float64, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    N.call("ipcb_collision_time", 0 if kind == "ee" else 1, n, N.ptr(a), N.ptr(b), N.ptr(t), N.ptr(status),
           N.stream_handle())
    return t, int(status.item())


def ee_collision_time(p_t0, p_t1, device="cuda"):
    return collision_time("ee", p_t0, p_t1, device)[0]


def pt_collision_time(p_t0, p_t1, device="cuda"):
    return collision_time("pt", p_t0, p_t1, device)[0]


def cubic_roots(coef, x0: float, x1: float, device="cuda"):
    """cubic_roots.py:96-193 on n cubics (coef ascending, (n, 4)) -> (n_roots, roots (n, 3), status)."""
    c = _dev(coef, device).reshape(-1, 4)
    n = c.shape[0]
    roots = torch.zeros((n, 3), dtype=torch.float64, device=device)
    nr = torch.zeros(n, dtype=torch.int32, device=device)
    status = torch.zeros(1, dtype=torch.int32, device=device)
    N.call("ipcb_cubic_roots", n, N.ptr(c), float(x0), float(x1), N.ptr(roots), N.ptr(nr), N.ptr(status),
           N.stream_handle())
    return nr, roots, int(status.item())
