"""Kernels of the Newton-Krylov finish and of the Anderson step.

* glide_dots / glide_combine against FP64 torch products (FP32 inputs:
  relative 1e-6 of the magnitude sum, FP64: 1e-13), bit-identical on repeat;
* glide_newton_rhs / glide_newton_update against a torch restatement (exact);
* glide_vanka_lu_masked: with the mask equal to the active set that
  glide_vanka_lu derives from f_H, the factors are bit-identical (cells at
  the switch itself excepted);
* the linear V-cycle (glide_linear_vcycle) cuts the linear residual
  |g + J d| / |g| on a dome state, and its CUDA-graph replay equals the eager
  call bit for bit;
* the Anderson step's native products equal torch FP64 products;
* the Newton-Krylov finish on the mixed and on the FP64 path takes Newton
  steps and reaches |r|/|r0| <= 1e-9 on the 128^2 dome, judged by the FP64
  oracle's own residual.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import random_state

pytestmark = pytest.mark.gpu


def _lib():
    from glide_b200 import _native as N
    return N.load(), N


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("k", [1, 4, 21, 32])
def test_dots_and_combine(dtype, k):
    lib, N = _lib()
    n = 100_003
    g = torch.Generator(device="cuda").manual_seed(k)
    V = torch.randn(k, n, generator=g, device="cuda", dtype=dtype)
    w = torch.randn(n, generator=g, device="cuda", dtype=dtype)
    out = torch.zeros(k, dtype=torch.float64, device="cuda")
    parts = torch.zeros(lib.glide_dots_parts(n) * 32, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    code = N.dtype_code(dtype)
    assert lib.glide_dots(code, n, k, V.data_ptr(), n, w.data_ptr(), out.data_ptr(), parts.data_ptr(), s) == 0
    ref = V.double() @ w.double()
    mag = V.double().abs() @ w.double().abs()
    tol = 1e-6 if dtype == torch.float32 else 1e-13
    assert torch.all((out - ref).abs() <= tol * mag)
    again = torch.zeros_like(out)
    assert lib.glide_dots(code, n, k, V.data_ptr(), n, w.data_ptr(), again.data_ptr(), parts.data_ptr(), s) == 0
    assert torch.equal(out, again)
    coef = torch.randn(k, generator=g, device="cuda", dtype=torch.float64)
    y = torch.randn(n, generator=g, device="cuda", dtype=dtype)
    y0 = y.clone()
    assert lib.glide_combine(code, n, k, V.data_ptr(), n, coef.data_ptr(), -0.5, y.data_ptr(), 1.0, s) == 0
    ref = y0.double() - 0.5 * (V.double().T @ coef)
    mag = y0.double().abs() + 0.5 * (V.double().abs().T @ coef.abs())
    assert torch.all((y.double() - ref).abs() <= (3e-6 if dtype == torch.float32 else 1e-14) * mag)
    assert lib.glide_dots(code, n, 33, V.data_ptr(), n, w.data_ptr(), out.data_ptr(), parts.data_ptr(), s) == -2


def _mixed_level(n=48, seed=3):
    from glide_b200.grid import Grid
    st = random_state(n=n, seed=seed)
    g = Grid(n, n, st["dx"], dt=st["dt"], dtype=torch.float64)
    for k in ("u", "v", "H", "bed", "B", "beta", "gamma", "f_u", "f_v", "f_H"):
        getattr(g, k).copy_(torch.as_tensor(st[k]))
    g.mask.zero_()
    return g, st


def test_newton_rhs_and_update():
    lib, N = _lib()
    g, st = _mixed_level()
    g.compute_residual()
    n, nU = g.n_total, g.nU
    rhs = torch.zeros(n, dtype=torch.float32, device="cuda")
    rraw = torch.zeros_like(rhs)
    mask = torch.zeros(g.ny, g.nx, dtype=torch.float32, device="cuda")
    a = g.level_args()
    s = torch.cuda.current_stream().cuda_stream
    assert lib.glide_newton_rhs(C.byref(a), g.r.data_ptr(), rhs.data_ptr(), rraw.data_ptr(), mask.data_ptr(), N.F32,
                                s) == 0
    act = (g.H - g.dt * g.r_H <= g.gamma)
    assert torch.equal(mask, act.float())
    ref = g.r.clone()
    ref[nU:] = torch.where(act.flatten(), (g.H - g.gamma).flatten(), g.r_H.flatten())
    assert torch.equal(rhs, ref.float())
    assert torch.equal(rraw, g.r.float())
    d = torch.randn(n, device="cuda", dtype=torch.float32) * 10
    base = g.U.clone()
    assert lib.glide_newton_update(C.byref(a), g.U.data_ptr(), base.data_ptr(), d.data_ptr(), N.F32, 0.5, s) == 0
    ref = base + 0.5 * d.double()
    ref[nU:] = torch.maximum(ref[nU:], g.gamma.flatten())
    assert torch.equal(g.U, ref)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_vanka_lu_masked_matches_residual_test(dtype):
    lib, N = _lib()
    from glide_b200.grid import Grid
    st = random_state(n=40, seed=9)
    g = Grid(40, 40, st["dx"], dt=st["dt"], dtype=dtype)
    for k in ("u", "v", "H", "bed", "B", "beta", "gamma", "f_u", "f_v", "f_H"):
        getattr(g, k).copy_(torch.as_tensor(st[k]))
    g.u.mul_(0.05)
    g.v.mul_(0.05)
    g.H.copy_(torch.where(torch.rand_like(g.H) < 0.2, g.gamma + 1e-3, g.H))
    g.mask.zero_()
    g.compute_residual()
    g.mask.copy_((g.H - g.dt * g.r_H <= g.gamma).to(dtype))
    a = g.level_args()
    s = torch.cuda.current_stream().cuda_stream
    lu1 = torch.zeros(25 * 1600, dtype=dtype, device="cuda")
    lu2 = torch.zeros_like(lu1)
    assert lib.glide_vanka_lu(C.byref(a), g.f_H.data_ptr(), lu1.data_ptr(), 0.0, s) == 0
    assert lib.glide_vanka_lu_masked(C.byref(a), lu2.data_ptr(), 0.0, s) == 0
    assert int(g.mask.sum()) > 0
    # cells away from the switch (the kernel's own local residual may round differently there)
    clear = ((g.H - g.dt * g.r_H - g.gamma).abs() > 1e-3).flatten()
    assert int(clear.sum()) > 0.9 * clear.numel()
    assert torch.equal(lu1.view(25, -1)[:, clear], lu2.view(25, -1)[:, clear])


def test_linear_vcycle_reduces_linear_residual_and_replays():
    lib, N = _lib()
    from glide_b200 import IcePhysics
    from glide_b200.synthetic import dome_case
    c = dome_case(1, n=64, dx=5000.0, n_levels=3)
    ph = IcePhysics(64, 64, c.dx, n_levels=3, thklim=c.thklim, precision="mixed", newton=True)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    ph.forward(c.dt, n_vcycles=1, update_geometry=False)
    nk = ph._newton_krylov()
    arr, nlev = nk.levels()
    cfg = ph.settings.native(ph.thklim)
    g64, g0 = ph.grid, ph.grids32[0]
    buf = g0.newton_buffers()
    s = torch.cuda.current_stream().cuda_stream
    a64 = g64.level_args()
    g64.compute_residual()
    assert lib.glide_newton_rhs(C.byref(a64), g64.r.data_ptr(), buf["lin_rhs"].data_ptr(), buf["r_raw"].data_ptr(),
                                buf["mask"].data_ptr(), N.F32, s) == 0
    assert lib.glide_convert(N.F32, g0.U.data_ptr(), g64.U.data_ptr(), g64.n_total, 0, s) == 0
    assert lib.glide_linear_setup(arr, nlev, C.byref(cfg), s) == 0
    assert lib.glide_linear_vcycle(arr, nlev, C.byref(cfg), s) == 0
    d_eager = buf["lin_d"].clone()
    # |g + J d| / |g| with the level-0 operator of the V-cycle
    rho = torch.zeros_like(buf["lin_rhs"])
    du, dv, dH = g0._vec_to_fields(d_eager)
    gu, gv, gH = g0._vec_to_fields(buf["lin_rhs"])
    ou, ov, oH = g0._vec_to_fields(rho)
    a0 = arr[0].a
    assert lib.glide_jvp_add(C.byref(a0), du.data_ptr(), dv.data_ptr(), dH.data_ptr(), gu.data_ptr(), gv.data_ptr(),
                             gH.data_ptr(), ou.data_ptr(), ov.data_ptr(), oH.data_ptr(), s) == 0
    red = float(rho.double().norm() / buf["lin_rhs"].double().norm())
    assert red < 0.5, red
    buf["lin_d"].zero_()
    assert lib.glide_graph_launch(nk.graph(cfg)[0], s) == 0
    torch.cuda.synchronize()
    assert torch.equal(buf["lin_d"], d_eager)
    nk.release()


def test_anderson_native_products_match_torch():
    from glide_b200.physics import _NativeProducts
    n = 50_001
    rows = torch.randn(4, n, dtype=torch.float64, device="cuda")
    w = torch.randn(n, dtype=torch.float64, device="cuda")
    p = _NativeProducts(n, torch.float64, "cuda")
    assert np.allclose(p.dots(rows, w), (rows @ w).cpu().numpy(), rtol=1e-12, atol=1e-12)
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    coef = np.array([0.5, -1.0, 2.0, 0.25])
    p.combine(rows, coef, out)
    assert torch.allclose(out, rows.T @ torch.as_tensor(coef, device="cuda"), rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_newton_krylov_finish_reaches_tolerance(precision):
    import bench
    from glide_b200 import IcePhysics
    from glide_b200.synthetic import dome_case
    from oracle.check import relative_residuals
    c = dome_case(2, n=128, dx=2500.0, n_levels=4)
    kw = dict(bench.FAST_KW if precision == "mixed" else bench.FP64_FAST_KW)
    kw.update(newton=True, newton_start=1e-1, newton_after=0, newton_min_gain=1.0, newton_local=2,
              newton_max_steps=12)
    ph = IcePhysics(128, 128, c.dx, n_levels=4, thklim=c.thklim, precision=precision,
                    settings=bench.fast_settings(), **kw)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    u, v, H = ph.forward(c.dt, tol=1e-9, max_vcycles=40, max_finish_sweeps=20000, update_geometry=False)
    info = ph.last_info
    assert info["newton_steps"] >= 1, info
    assert info["rel_residual"] <= 1e-9, info
    geo = dict(bed=c.bed, B=c.B, beta=c.beta, H_prev=c.thickness, smb=c.smb, dx=c.dx, dt=c.dt, thklim=c.thklim)
    state = tuple(t.detach().double().cpu().numpy() for t in (u, v, H))
    orc = relative_residuals([(geo, [state])], workers=1)[0][0]
    assert orc <= 1.05e-9, (orc, info)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_adjoint_fgmres_matches_cycles_and_sweeps(precision):
    """The adjoint multiplier by FGMRES (adjoint V-cycle preconditioner) and by
    the reference's cycles followed by fine-level adjoint sweeps solve the same
    system J_m^T lam = f: both reach 1e-10 and their gradients agree to
    1e-7 relative.  FGMRES needs far fewer fine-level operator applications."""
    import bench
    from glide_b200 import IcePhysics
    from glide_b200.synthetic import dome_case
    c = dome_case(2, n=128, dx=2500.0, n_levels=4)
    kw = dict(bench.FAST_KW if precision == "mixed" else bench.FP64_FAST_KW)
    grads, infos = [], []
    for krylov in (30, 0):
        ph = IcePhysics(128, 128, c.dx, n_levels=4, thklim=c.thklim, precision=precision,
                        settings=bench.fast_settings(), adjoint_krylov=krylov, **kw)
        ph.set_geometry(c.bed, c.thickness)
        ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
        ph.forward(c.dt, tol=1e-10, max_vcycles=40, max_finish_sweeps=20000, update_geometry=False)
        assert ph.last_info["rel_residual"] <= 1e-10, ph.last_info
        gen = torch.Generator().manual_seed(3)
        g = ph.grid
        cu = torch.randn(tuple(g.u.shape), generator=gen, dtype=torch.float64).cuda()
        cv = torch.randn(tuple(g.v.shape), generator=gen, dtype=torch.float64).cuda()
        grads.append(ph.adjoint(cu, cv, torch.zeros_like(g.H), tol=1e-10, max_vcycles=100,
                                max_finish_sweeps=40000).double().clone())
        infos.append(dict(ph.last_adjoint_info))
        assert infos[-1]["rel_residual"] <= 1e-10, infos[-1]
    assert infos[0].get("krylov_its", 0) >= 1 and "krylov_rel_residual" not in infos[0], infos[0]
    assert infos[0]["krylov_its"] <= 300, infos[0]
    rel = float((grads[0] - grads[1]).norm() / grads[1].norm())
    assert rel <= 1e-7, (rel, infos)
