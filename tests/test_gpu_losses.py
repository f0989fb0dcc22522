"""Fused loss kernels vs the torch expressions of the reference's helpers
(glide/physics.py:262-411): abs and Huber misfit with NaN observations, their
gradients, and the Tikhonov term and gradient.  FP64: losses within 1e-12,
gradients within 1e-13 (norm-wise relative; only the summation order
differs).  FP32: 1e-5 (the fused kernels sum in FP64)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = torch.as_tensor(a).double().cpu(), torch.as_tensor(b).double().cpu()
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b).clamp_min(1e-300)).item()


def _fields(dtype, ny=37, nx=53):
    g = torch.Generator().manual_seed(3)
    u = torch.randn(ny, nx + 1, generator=g, dtype=torch.float64) * 50
    v = torch.randn(ny + 1, nx, generator=g, dtype=torch.float64) * 50
    uo = u + torch.randn(ny, nx + 1, generator=g, dtype=torch.float64) * 5
    vo = v + torch.randn(ny + 1, nx, generator=g, dtype=torch.float64) * 5
    uo[3, 4] = float("nan")
    vo[10, :7] = float("nan")
    uo[5, 6] = u[5, 6]  # an exact zero difference
    return [t.to(dtype=dtype, device="cuda") for t in (u, v, uo, vo)]


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("kind", ["abs", "huber"])
def test_fused_misfit_matches_reference_helpers(dtype, kind):
    from glide_b200.losses import misfit
    from glide_b200.physics import abs_grad, abs_loss, huber_grad, huber_loss
    u, v, uo, vo = _fields(dtype)
    L, gu, gv = misfit(u, v, uo, vo, kind=kind, eps=10.0)
    if kind == "abs":
        Lr, (gur, gvr) = abs_loss(u, v, uo, vo), abs_grad(u, v, uo, vo)
    else:
        Lr, (gur, gvr) = huber_loss(u, v, uo, vo, eps=10.0), huber_grad(u, v, uo, vo, eps=10.0)
    tl, tg = (1e-12, 1e-13) if dtype == torch.float64 else (1e-5, 1e-5)
    assert abs(float(L) - float(Lr)) <= tl * abs(float(Lr))
    assert _rel(gu, gur) <= tg and _rel(gv, gvr) <= tg
    assert torch.isfinite(gu).all() and torch.isfinite(gv).all()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_fused_tikhonov_matches_reference_helper(dtype):
    from glide_b200.losses import tikhonov
    from glide_b200.physics import tikhonov_regularization
    f = torch.as_tensor(np.random.default_rng(4).random((29, 41)), dtype=dtype, device="cuda")
    L, g = tikhonov(f)
    Lr, gr = tikhonov_regularization(f)
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    assert abs(float(L) - Lr) <= tol * abs(Lr)
    assert _rel(g, gr) <= max(tol, 1e-13)
