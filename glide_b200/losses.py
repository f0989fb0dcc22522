"""Fused loss kernels of the inverse problem (glide/physics.py:262-411).

``misfit`` returns the abs or Huber velocity misfit and its gradient from one
kernel pass (NaN differences count as 0, both gradients divided by the number
of u entries, as the reference's helpers do); ``tikhonov`` returns the
neighbour-difference regulariser and its gradient.  Losses are 0-d FP64
device tensors (no host synchronisation); the gradients have the inputs'
dtype.  The torch expressions in ``glide_b200.physics`` are the same
formulas, kept as the reference-named helpers.
"""
from __future__ import annotations

import torch

from . import _native as N

KINDS = {"abs": 0, "huber": 1}


def _parts(n, device):
    return torch.empty(N.load().glide_loss_parts(int(n)), dtype=torch.float64, device=device)


def misfit(u, v, u_obs, v_obs, kind="huber", eps=10.0):
    """(L, dL/du, dL/dv) with L = L_u + L_v (abs or Huber)."""
    u, v = u.contiguous(), v.contiguous()
    u_obs = u_obs.to(dtype=u.dtype).contiguous()
    v_obs = v_obs.to(dtype=v.dtype).contiguous()
    gu, gv = torch.empty_like(u), torch.empty_like(v)
    out = torch.empty(3, dtype=torch.float64, device=u.device)
    N.check(N.load().glide_misfit(N.dtype_code(u.dtype), KINDS[kind], float(eps), u.data_ptr(), v.data_ptr(),
                                  u_obs.data_ptr(), v_obs.data_ptr(), u.numel(), v.numel(), gu.data_ptr(),
                                  gv.data_ptr(), out.data_ptr(), _parts(max(u.numel(), v.numel()), u.device).data_ptr(),
                                  N.stream_handle()), "misfit")
    return out[0], gu, gv


def tikhonov(field):
    """(1/2 sum of squared neighbour differences, gradient) of an (ny, nx) field."""
    f = field.contiguous()
    ny, nx = f.shape
    g = torch.empty_like(f)
    out = torch.empty(1, dtype=torch.float64, device=f.device)
    N.check(N.load().glide_tikhonov(N.dtype_code(f.dtype), f.data_ptr(), ny, nx, g.data_ptr(), out.data_ptr(),
                                    _parts(f.numel(), f.device).data_ptr(), N.stream_handle()), "tikhonov")
    return out[0], g
