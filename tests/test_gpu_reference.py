"""FP32 kernels vs the reference's own CUDA kernels on the same inputs.

The reference kernels are built from the reference tree into
``oracle/_ref/libglide_ref.so`` (``oracle/build_ref.py``) and travel with the
repository snapshot; the test is skipped when that library is absent.
Tolerances (norm-wise relative error, FP32 vs FP32 fast-math):
  single operators <= 2e-5; one Vanka sweep <= 1e-4; one forward step
  (1 V-cycle, reference settings, 64^2 dome) <= 1e-6 -- measured 1.8e-7 (u),
  1.7e-7 (v), 3.3e-8 (H) on a B200.
"""
import numpy as np
import pytest

from conftest import random_state

pytestmark = pytest.mark.gpu


def _ref():
    from oracle import ref_replay as R
    if not R.available():
        pytest.skip("reference kernels not built (oracle/_ref)")
    return R


def rel(a, b):
    a = a.double().cpu().numpy() if hasattr(a, "cpu") else np.asarray(a, float)
    b = b.double().cpu().numpy() if hasattr(b, "cpu") else np.asarray(b, float)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _pair(shape, seed, gl=False):
    import torch
    from glide_b200.grid import Grid
    R = _ref()
    ny, nx = shape
    n = max(ny, nx)
    st = random_state(n=n, seed=seed)
    for k in list(st):
        if isinstance(st[k], np.ndarray):
            a = st[k]
            st[k] = np.ascontiguousarray(a[:ny + a.shape[0] - n, :nx + a.shape[1] - n]).astype(np.float32)
    mine = Grid(ny, nx, st["dx"], dt=st["dt"], dtype=torch.float32, gl_derivatives=gl)
    ref = R.RefGrid(ny, nx, st["dx"], st["dt"], gl_derivatives=gl)
    for g in (mine, ref):
        for k in ("u", "v", "H", "bed", "B", "beta", "mask", "gamma", "f_u", "f_v", "f_H", "d_u", "d_v", "d_H"):
            getattr(g, k).copy_(torch.as_tensor(st[k]))
    return mine, ref


@pytest.mark.parametrize("shape", [(64, 64), (60, 100)])
def test_residual_jvp_vjp_grad(shape):
    mine, ref = _pair(shape, 21)
    for g in (mine, ref):
        g.compute_residual()
        g.compute_jvp()
        g.lambda_u.copy_(g.f_u)
        g.lambda_v.copy_(g.f_v)
        g.lambda_H.copy_(g.f_H)
        g.compute_vjp()
    for a in ("r_u", "r_v", "r_H", "j_u", "j_v", "j_H", "l_u", "l_v", "l_H"):
        assert rel(getattr(mine, a), getattr(ref, a)) <= 2e-5, a
    for g in (mine, ref):
        g.lambda_u.copy_(g.d_u)
        g.lambda_v.copy_(g.d_v)
    assert rel(mine.compute_grad_beta(), ref.compute_grad_beta()) <= 2e-5


@pytest.mark.parametrize("local", [False, True])
def test_vanka_sweep(local):
    import torch
    mine, ref = _pair((64, 64), 22)
    em = torch.zeros((64, 64), device="cuda")
    em[5, 40] = 1
    em[30, 13] = 1
    for g in (mine, ref):
        g.u.mul_(0.02)
        g.v.mul_(0.02)
        g.error_mask.copy_(em)
    u0, v0, H0 = mine.u.clone(), mine.v.clone(), mine.H.clone()
    if local:
        mine.vanka_sweep_local(1)
        ref.vanka_sweep_local(1)
    else:
        mine.vanka_sweep(1)
        ref.vanka_sweep(1)
    assert rel(mine.u - u0, ref.u - u0) <= 1e-4
    assert rel(mine.v - v0, ref.v - v0) <= 1e-4
    assert rel(mine.H - H0, ref.H - H0) <= 1e-4


def test_forward_step_vs_reference():
    from glide_b200 import IcePhysics
    from glide_b200.synthetic import dome_case
    R = _ref()
    c = dome_case(0, n=64, dx=5000.0, n_levels=3)
    mine = IcePhysics(64, 64, c.dx, n_levels=3, thklim=c.thklim, precision="fp32")
    ref = R.RefIcePhysics(64, 64, c.dx, n_levels=3, thklim=c.thklim)
    for ph in (mine, ref):
        ph.set_geometry(c.bed, c.thickness)
        ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    a = mine.forward(c.dt, n_vcycles=1)
    b = ref.forward(c.dt, n_vcycles=1)
    errs = [rel(x, y) for x, y in zip(a, b)]
    print("forward step vs reference kernels (u, v, H):", errs)
    for e in errs:
        assert e <= 1e-6
