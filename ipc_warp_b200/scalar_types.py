"""Precision switch (scalar_types.py:1-43 of the reference).

``USE_FLOAT32`` selects the scalar type of positions, contact records,
triplet values and forces.  Set the environment variable ``IPCB_FP64=1``
before import (or call :func:`set_float32`) for the double build that serves
as the error reference.  Whatever the switch, the float32 closest-point
distances decide candidates and gates, as in the reference (its DCD casts
every position through ``wp.vec3``), the barrier and geometry run in double,
and energies are accumulated in double.
"""
from __future__ import annotations

import os

import torch

USE_FLOAT32 = os.environ.get("IPCB_FP64", "0") not in ("1", "true", "True")


def set_float32(flag: bool) -> None:
    global USE_FLOAT32
    USE_FLOAT32 = bool(flag)


def scalar() -> torch.dtype:
    return torch.float32 if USE_FLOAT32 else torch.float64


def scalar_epsilon() -> float:
    return 1.1920928955078125e-7 if USE_FLOAT32 else 2.220446049250313e-16
