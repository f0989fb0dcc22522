"""FP64 oracle residual of solved states, on the host cores.

Test and bench-checker infrastructure only: nothing in the product imports
it.  For a geometry and a list of states (u, v, H) it evaluates the residual
norm the tolerance solver stops on,

    |r| = sqrt(|r_u|^2 + |r_v|^2 + |FB(r_H, H - gamma)|^2)

(glide/physics.py:176-198, FB as glide/grid.py:205-208), with the FP64
NumPy restatement of compute_residual (``oracle.ssa.residual``), f_u = f_v = 0,
f_H = H_prev / dt + smb (glide/physics.py:173), gamma = thklim and no active
mask, so that a state's |r| / |r0| (r0: the residual of the step's starting
state u = v = 0, H = H_prev) is judged by the oracle's own arithmetic.
Geometries are spread over worker processes started with ``spawn``.
"""
from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np

from . import ssa
from .ssa import Params


def residual_parts(u, v, H, bed, B, beta, H_prev, smb, dx, dt, thklim=0.1, p: Params | None = None):
    """Sums of squares (r_u, r_v, FB(r_H, H - gamma)) of one state."""
    p = p or Params()
    zeros_u, zeros_v = np.zeros_like(u), np.zeros_like(v)
    gamma = np.full_like(H, thklim)
    f_H = H_prev / dt + smb
    ru, rv, rH = ssa.residual(u, v, H, zeros_u, zeros_v, f_H, bed, B, beta, np.zeros_like(H), gamma, p, dx, dt)
    a, b = rH, H - gamma
    fb = a + b - np.sqrt(a * a + b * b)
    return float(np.sum(ru * ru)), float(np.sum(rv * rv)), float(np.sum(fb * fb))


def _job(args):
    geo, states = args
    out = []
    for st in states:
        if st is None:   # the step's starting state
            ny, nx = geo["H_prev"].shape
            st = (np.zeros((ny, nx + 1)), np.zeros((ny + 1, nx)), geo["H_prev"])
        out.append(residual_parts(*st, geo["bed"], geo["B"], geo["beta"], geo["H_prev"], geo["smb"], geo["dx"],
                                  geo["dt"], geo["thklim"]))
    return out


def relative_residuals(jobs, workers=None):
    """``jobs``: list of (geometry dict with bed, B, beta, H_prev, smb, dx, dt,
    thklim; list of states (u, v, H) as float64 arrays).  Returns per job the
    list of |r| / |r0| of its states, r0 being the starting state's residual."""
    workers = max(1, min(int(workers or os.cpu_count() or 1), len(jobs)))
    tasks = [(geo, [None] + list(states)) for geo, states in jobs]
    if workers > 1:
        with mp.get_context("spawn").Pool(workers) as pool:
            parts = pool.map(_job, tasks)
    else:
        parts = [_job(t) for t in tasks]
    out = []
    for p in parts:
        r0 = float(np.sqrt(sum(p[0])))
        out.append([float(np.sqrt(sum(q))) / r0 if r0 > 0 else 0.0 for q in p[1:]])
    return out
