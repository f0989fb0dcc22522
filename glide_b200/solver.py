"""FASCD and adjoint V-cycles (glide/solver.py:1-220) on the native driver.

``fascd_vcycle(grid, thklim, finest=False)`` and ``adjoint_vcycle(grid)``
keep the reference signatures; one call issues the whole cycle on the
current CUDA stream through ``glide_fascd_vcycle`` / ``glide_adjoint_vcycle``
(no host synchronisation inside).  Extra keyword arguments expose the
smoother settings the reference hard-codes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _native as N


@dataclass
class SolverSettings:
    """Smoother/cycle settings; the defaults are the reference's values
    (glide/solver.py:96,109,144,147-155,177,183; glide/grid.py:305-317;
    glide/cuda/vanka.cu:406-416)."""
    n_coarse: int = 200        # coarsest-level sweeps
    n_smooth: int = 10         # pre/post sweeps
    n_local_outer: int = 10    # error-driven local smoothing rounds
    n_local: int = 10          # local sweeps per round
    n_newton: int = 10         # local Newton iterations per sweep
    omega: float = 0.5         # U += omega * delta
    shift: float = 1.0         # diagonal shift of the local Newton matrix
    err_threshold: float = 0.01  # local error indicator threshold
    adj_coarse: int = 100
    adj_smooth: int = 10
    adj_omega: float = 1.0
    exact_adjoint: bool = False  # reference VJP/grad boundary handling when False
    smooth_H_correction: bool = False  # bilinear instead of injected coarse H correction
    newton_step: float = 0.25  # fraction of each local Newton step (relaxation_factor, glide/cuda/vanka.cu:416)
    coarse_line_search: bool = False  # finest-level step on the coarse correction (reference: full step)
    pivoted_lu: bool = False   # row-pivoted local solves (glide/cuda/common.cu:180-233; unused by the reference)
    # linear V-cycle of the Newton-Krylov finishing solver (no counterpart in the reference)
    lin_pre: int = 2           # linear Vanka sweeps before the coarse correction
    lin_post: int = 2          # ... and after it
    lin_coarse: int = 20       # linear sweeps on the coarsest level
    lin_omega: float = 0.5     # damping of each linear sweep
    lin_shift: float = 0.0     # diagonal shift of the local factors
    # adjoint active set: H <= gamma + adj_active_tol (glide/grid.py:332-334 uses 0.1 m)
    adj_active_tol: float = 0.1

    def native(self, thklim) -> N.SolverConfig:
        c = N.SolverConfig()
        c.thklim = float(thklim)
        c.n_coarse, c.n_smooth, c.n_local_outer, c.n_local, c.n_newton = (
            self.n_coarse, self.n_smooth, self.n_local_outer, self.n_local, self.n_newton)
        c.omega, c.shift, c.err_threshold = float(self.omega), float(self.shift), float(self.err_threshold)
        c.adj_coarse, c.adj_smooth, c.adj_omega = self.adj_coarse, self.adj_smooth, float(self.adj_omega)
        c.exact_adjoint = int(self.exact_adjoint)
        c.smooth_H_correction = int(self.smooth_H_correction)
        c.newton_step = float(self.newton_step)
        c.coarse_line_search = int(self.coarse_line_search)
        c.pivoted_lu = int(self.pivoted_lu)
        c.lin_pre, c.lin_post, c.lin_coarse = int(self.lin_pre), int(self.lin_post), int(self.lin_coarse)
        c.lin_omega, c.lin_shift = float(self.lin_omega), float(self.lin_shift)
        c.adj_active_tol = float(self.adj_active_tol)
        return c


REFERENCE = SolverSettings()


def hierarchy(grid):
    out = [grid]
    while out[-1].child is not None:
        out.append(out[-1].child)
    return out


def native_levels(grid):
    gs = hierarchy(grid)
    arr = (N.Level * len(gs))()
    for k, g in enumerate(gs):
        arr[k] = g.native_level()
    return arr, len(gs)


def restrict_parameters(grid):
    """bed, B, beta, H_prev, smb to the child (glide/solver.py:53-61)."""
    if grid.child is None:
        return
    arr, n = native_levels(grid)
    lib = N.load()
    # restrict only this level pair
    sub = (N.Level * 2)(arr[0], arr[1])
    N.check(lib.glide_restrict_parameters(sub, 2, 0, N.stream_handle()), "restrict parameters")


def restrict_parameters_to_hierarchy(grid):
    """glide/solver.py:64-68."""
    if grid.child is None:
        return
    arr, n = native_levels(grid)
    N.check(N.load().glide_restrict_parameters(arr, n, 0, N.stream_handle()), "restrict parameters")


def fascd_vcycle(grid, thklim, finest=False, settings: SolverSettings = REFERENCE):
    """One FASCD V-cycle (glide/solver.py:71-157)."""
    arr, n = native_levels(grid)
    cfg = settings.native(thklim)
    N.check(N.load().glide_fascd_vcycle(arr, n, 0, int(bool(finest)), C.byref(cfg), N.stream_handle()),
            "fascd_vcycle")


def adjoint_vcycle(grid, settings: SolverSettings = REFERENCE, thklim=0.1):
    """One adjoint V-cycle (glide/solver.py:160-220)."""
    arr, n = native_levels(grid)
    cfg = settings.native(thklim)
    N.check(N.load().glide_adjoint_vcycle(arr, n, 0, C.byref(cfg), N.stream_handle()), "adjoint_vcycle")
