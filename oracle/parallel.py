"""Row-strip parallel evaluation of the oracle's Vanka sweep on host cores.

Test / CPU-baseline infrastructure.  One reference Vanka launch is a Jacobi
update (every cell reads the same input state), so cell rows can be split
into strips that are solved independently; each strip carries a 3-row halo,
enough for every stencil read of its own rows (eta needs u/v two rows away),
so strip interiors are identical to the whole-grid oracle.  Workers are
started with the ``spawn`` method.
"""
from __future__ import annotations

import multiprocessing as mp
import os

import numpy as np

from .ssa import Params
from .vanka import vanka_deltas

HALO = 3


def _strip(args):
    (u, v, H, f_u, f_v, f_H, bed, B, beta, gamma, p, dx, dt, n_newton, shift, r0, r1, ny) = args
    return r0, r1, vanka_deltas(u, v, H, f_u, f_v, f_H, bed, B, beta, gamma, p, dx, dt, n_newton, shift=shift,
                                return_cells=True)


def _cut(a, lo, hi, extra):
    return np.ascontiguousarray(a[lo:hi + extra])


class ParallelSweeper:
    """Evaluate one Vanka sweep's deltas with ``workers`` processes."""

    def __init__(self, workers=None):
        self.workers = int(workers or os.cpu_count() or 1)
        self._pool = mp.get_context("spawn").Pool(self.workers) if self.workers > 1 else None

    def close(self):
        if self._pool is not None:
            self._pool.close()
            self._pool.join()
            self._pool = None

    def deltas(self, u, v, H, f_u, f_v, f_H, bed, B, beta, gamma, p: Params, dx, dt, n_newton=10, shift=1.0):
        """Same result as ``vanka_deltas`` (face-summed du, dv and dH)."""
        ny, nx = H.shape
        bounds = np.linspace(0, ny, self.workers + 1).astype(int)
        jobs = []
        for a, b in zip(bounds[:-1], bounds[1:]):
            if b <= a:
                continue
            lo, hi = max(a - HALO, 0), min(b + HALO, ny)
            # a strip is a smaller grid: exact for rows >= HALO from a cut that is
            # not a domain edge (clamping and boundary rules act only at true edges)
            jobs.append((_cut(u, lo, hi, 0), _cut(v, lo, hi, 1), _cut(H, lo, hi, 0), _cut(f_u, lo, hi, 0),
                         _cut(f_v, lo, hi, 1), _cut(f_H, lo, hi, 0), _cut(bed, lo, hi, 0), _cut(B, lo, hi, 0),
                         _cut(beta, lo, hi, 0), _cut(gamma, lo, hi, 0), p, dx, dt, n_newton, shift, a - lo, b - lo, ny))
        results = self._pool.map(_strip, jobs) if self._pool is not None else [_strip(j) for j in jobs]
        cells = [np.zeros((ny, nx)) for _ in range(5)]
        row = 0
        for (r0, r1, parts), (a, b) in zip(results, [(x, y) for x, y in zip(bounds[:-1], bounds[1:]) if y > x]):
            for k in range(5):
                cells[k][a:b] = parts[k][r0:r1]
        d_ul, d_ur, d_vt, d_vb, dH = cells
        du = np.zeros((ny, nx + 1))
        dv = np.zeros((ny + 1, nx))
        du[:, :nx] += d_ul
        du[:, 1:] += d_ur
        dv[:ny, :] += d_vt
        dv[1:, :] += d_vb
        return du, dv, dH
