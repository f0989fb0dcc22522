"""Kernel access and multigrid transfer operators (glide/kernels.py:1-236).

Same function names and call signatures as the reference:
``restrict_vfacet(u_fine, kernels, u_coarse=None)`` and friends take and
return device tensors; ``get_kernels()`` returns the loaded native library
(the reference returns its CuPy RawModule container);
``make_physics_params`` builds the parameter struct.
"""
from __future__ import annotations

import torch

from . import _native as N


class Kernels:
    """Handle on the native library (the reference compiles CuPy modules)."""

    def __init__(self):
        self.lib = N.load()

    def version(self) -> str:
        return self.lib.glide_version().decode()


_kernels = None


def get_kernels() -> Kernels:
    global _kernels
    if _kernels is None:
        _kernels = Kernels()
    return _kernels


def make_physics_params(n=3.0, eps_reg=1e-5, water_drag=0.001, calving_rate=1.0, gl_sigmoid_c=0.1,
                        gl_derivatives=False) -> N.PhysicsParams:
    """Parameter struct of the C ABI (glide/kernels.py:10-49)."""
    return N.PhysicsParams(float(n), float(eps_reg), float(water_drag), float(calving_rate), float(gl_sigmoid_c),
                           int(bool(gl_derivatives)))


def _batch(t, rows_extra, cols_extra):
    if t.dim() == 2:
        return 1, t.shape[0] - rows_extra, t.shape[1] - cols_extra
    return t.shape[0], t.shape[1] - rows_extra, t.shape[2] - cols_extra


def _restrict(field, use_max, fine, coarse, kernels):
    lib = (kernels or get_kernels()).lib
    re, ce = (0, 1) if field == 0 else ((1, 0) if field == 1 else (0, 0))
    nb, ny, nx = _batch(fine, re, ce)
    nyc, nxc = ny // 2, nx // 2
    if coarse is None:
        shape = (nyc + re, nxc + ce) if nb == 1 and fine.dim() == 2 else (nb, nyc + re, nxc + ce)
        coarse = torch.empty(shape, dtype=fine.dtype, device=fine.device)
    fine = fine.contiguous()
    N.check(lib.glide_restrict(N.dtype_code(fine.dtype), field, int(use_max), fine.data_ptr(), coarse.data_ptr(),
                               nyc, nxc, nb, N.stream_handle()), "restrict")
    return coarse


def restrict_vfacet(u_fine, kernels=None, u_coarse=None):
    """Tangential 2-average of u (glide/kernels.py:90-107)."""
    return _restrict(0, 0, u_fine, u_coarse, kernels)


def restrict_hfacet(v_fine, kernels=None, v_coarse=None):
    """glide/kernels.py:110-127."""
    return _restrict(1, 0, v_fine, v_coarse, kernels)


def restrict_cell_centered(f_fine, kernels=None, f_coarse=None):
    """4-cell average (glide/kernels.py:130-146)."""
    return _restrict(2, 0, f_fine, f_coarse, kernels)


def restrict_max_pool(f_fine, kernels=None, f_coarse=None):
    """glide/kernels.py:149-165."""
    return _restrict(2, 1, f_fine, f_coarse, kernels)


def _prolong(field, smooth, coarse, fine, kernels, add=False):
    lib = (kernels or get_kernels()).lib
    re, ce = (0, 1) if field == 0 else ((1, 0) if field == 1 else (0, 0))
    nb, nyc, nxc = _batch(coarse, re, ce)
    if fine is None:
        shape = (2 * nyc + re, 2 * nxc + ce) if coarse.dim() == 2 else (nb, 2 * nyc + re, 2 * nxc + ce)
        fine = torch.empty(shape, dtype=coarse.dtype, device=coarse.device)
    coarse = coarse.contiguous()
    N.check(lib.glide_prolong(N.dtype_code(coarse.dtype), field, int(bool(smooth)), int(add), coarse.data_ptr(),
                              fine.data_ptr(), nyc, nxc, nb, N.stream_handle()), "prolong")
    return fine


def prolongate_vfacet(u_coarse, kernels=None, u_fine=None, smooth=True):
    """glide/kernels.py:168-189 (bilinear when smooth, else linear-normal)."""
    return _prolong(0, smooth, u_coarse, u_fine, kernels)


def prolongate_hfacet(v_coarse, kernels=None, v_fine=None, smooth=True):
    """glide/kernels.py:192-213."""
    return _prolong(1, smooth, v_coarse, v_fine, kernels)


def prolongate_cell_centered(H_coarse, kernels=None, H_fine=None, smooth=True):
    """glide/kernels.py:216-236 (bilinear when smooth, else injection)."""
    return _prolong(2, smooth, H_coarse, H_fine, kernels)
