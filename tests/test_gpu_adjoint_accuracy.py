"""Accuracy of the mixed-precision adjoint against the FP64 oracle.

The mixed path solves the adjoint J_m^T lambda = -dL/dU with FP32 adjoint
V-cycles as the correction solver of the FP64 adjoint residual (J_m: rows of
cells at the thickness limit replaced by the identity, as the reference's
adjoint smoother sees them).  At one converged forward state of the
64x64 dome (dx = 5 km, 3 levels, the plain-method configuration) and of one
1024x1024 benchmark geometry, its grad_beta, solved to |r_adj| / |f_adj| <=
1e-8, must lie within 1e-6 relative (2-norm) of the FP64 adjoint gradient:

* 64^2: the FP64 NumPy oracle's own adjoint V-cycles (glide/solver.py:160-220
  restated), iterated until the oracle's adjoint residual is below 1e-12 of
  |f_adj|, then its grad_beta (glide/cuda/grad.cu:1-74 restated);
* 1024^2: the FP64 GPU adjoint solved to 1e-10 (its kernels match the oracle
  to 1e-10 per operator in test_gpu_kernels.py), whose multiplier the oracle
  checks: the oracle's VJP gives |f_adj - J_m^T lambda| / |f_adj| <= 1e-10.

The loss is L = 1/2 |u - u_obs|^2 + 1/2 |v - v_obs|^2 with (u_obs, v_obs)
the forward answer for beta scaled by 1.3.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().double().cpu().numpy()


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _solved(case, precision, beta_scale=1.0, tol=1e-10, **kw):
    import bench
    from glide_b200 import IcePhysics
    if precision == "mixed":
        kw = dict(settings=bench.fast_settings(), **bench.FAST_KW, **kw)
    else:
        kw = dict(settings=bench.fast_settings(), **bench.FP64_FAST_KW, **kw)
    ph = IcePhysics(case.ny, case.nx, case.dx, n_levels=case.n_levels, thklim=case.thklim, precision=precision,
                    **kw)
    ph.set_geometry(case.bed, case.thickness)
    ph.set_parameters(B=case.B, beta=case.beta * beta_scale, smb=case.smb)
    ph.forward(case.dt, tol=tol, max_vcycles=60, update_geometry=False, max_finish_sweeps=20000)
    assert ph.last_info["rel_residual"] <= tol, ph.last_info
    return ph


def _cotangent(case, ph):
    obs = _solved(case, "fp64", beta_scale=1.3, tol=1e-6)
    du = (ph.grid.u - obs.grid.u).detach().clone()
    dv = (ph.grid.v - obs.grid.v).detach().clone()
    return du, dv


def _oracle_adjoint(case, ph, du, dv, tol=1e-12, max_cycles=400):
    """The oracle's adjoint V-cycles at the GPU's converged state (coarse
    levels linearised at the restricted state), to |r_adj| <= tol |f_adj|."""
    from oracle.multigrid import (OracleIcePhysics, adjoint_vcycle, restrict_cell, restrict_u, restrict_v)
    orc = OracleIcePhysics(case.ny, case.nx, case.dx, n_levels=case.n_levels, thklim=case.thklim)
    orc.set_geometry(case.bed, case.thickness)
    orc.set_parameters(B=case.B, beta=case.beta, smb=case.smb)
    g = orc.grid
    for lv in orc.grids:
        lv.dt = case.dt
    g.u, g.v, g.H = _np(ph.grid.u), _np(ph.grid.v), _np(ph.grid.H)
    for par, ch in zip(orc.grids[:-1], orc.grids[1:]):
        ch.u, ch.v, ch.H = restrict_u(par.u), restrict_v(par.v), restrict_cell(par.H)
    g.fa_u, g.fa_v, g.fa_H = -_np(du), -_np(dv), np.zeros_like(g.H)
    g.lu, g.lv, g.lH = np.zeros_like(g.u), np.zeros_like(g.v), np.zeros_like(g.H)
    f0 = np.sqrt(np.sum(g.fa_u ** 2) + np.sum(g.fa_v ** 2))
    rel = 1.0
    for _ in range(max_cycles):
        adjoint_vcycle(g)
        g.compute_mask()
        ru, rv, rH = g.adjoint_residual()
        g.mask = np.zeros_like(g.mask)
        rel = np.sqrt(np.sum(ru ** 2) + np.sum(rv ** 2) + np.sum(rH ** 2)) / f0
        if rel <= tol:
            break
    return g.compute_grad_beta(), rel


def test_mixed_adjoint_vs_oracle_64():
    from glide_b200.synthetic import dome_case
    c = dome_case(0, n=64, dx=5000.0, n_levels=3)
    ph = _solved(c, "mixed")
    du, dv = _cotangent(c, ph)
    g_mixed = ph.adjoint(du, dv, torch.zeros_like(ph.grid.H), tol=1e-8, max_vcycles=100)
    assert ph.last_adjoint_info["rel_residual"] <= 1e-8
    g_orc, rel_orc = _oracle_adjoint(c, ph, du, dv)
    assert rel_orc <= 1e-12, rel_orc
    err = _rel(_np(g_mixed), g_orc)
    assert err <= 1e-6, err


def test_mixed_adjoint_vs_fp64_1024():
    import bench
    from oracle import ssa
    c = bench.make_cases(1024, [5])[0]
    ph = _solved(c, "mixed", tol=1e-6)   # both adjoints linearise at this same state
    du, dv = _cotangent(c, ph)
    zero = torch.zeros_like(ph.grid.H)
    g_mixed = _np(ph.adjoint(du, dv, zero, tol=1e-8, max_vcycles=100))
    assert ph.last_adjoint_info["rel_residual"] <= 1e-8
    # FP64 adjoint at the same state
    from glide_b200 import IcePhysics
    ref = IcePhysics(c.ny, c.nx, c.dx, n_levels=c.n_levels, thklim=c.thklim, precision="fp64",
                     settings=bench.fast_settings(), **bench.FP64_FAST_KW)
    ref.set_geometry(c.bed, c.thickness)
    ref.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    ref._set_dt(c.dt)
    ref.grid.U.copy_(ph.grid.U)
    ref.grid.f_H.copy_(ph.grid.f_H)
    from glide_b200.kernels import restrict_cell_centered, restrict_hfacet, restrict_vfacet
    for par, ch in zip(ref.grids[:-1], ref.grids[1:]):   # coarse levels linearised at the restricted state
        restrict_vfacet(par.u, u_coarse=ch.u)
        restrict_hfacet(par.v, v_coarse=ch.v)
        restrict_cell_centered(par.H, f_coarse=ch.H)
    g_ref = _np(ref.adjoint(du, dv, zero, tol=1e-10, max_vcycles=200, max_finish_sweeps=10000))
    assert ref.last_adjoint_info["rel_residual"] <= 1e-10, ref.last_adjoint_info
    # the oracle checks the FP64 multiplier: |f_adj - J_m^T lambda| / |f_adj|
    u, v, H = _np(ref.grid.u), _np(ref.grid.v), _np(ref.grid.H)
    lu, lv, lH = _np(ref.grid.lambda_u), _np(ref.grid.lambda_v), _np(ref.grid.lambda_H)
    gamma = np.full_like(H, c.thklim)
    mask = (H <= gamma + 0.1).astype(float)
    vu, vv, vH = ssa.vjp(u, v, H, lu, lv, lH, c.bed, c.B, c.beta, mask, gamma, ssa.Params(), c.dx, c.dt)
    fu, fv = -_np(du), -_np(dv)
    r = np.sqrt(np.sum((fu - vu) ** 2) + np.sum((fv - vv) ** 2) + np.sum(vH ** 2))
    assert r / np.sqrt(np.sum(fu ** 2) + np.sum(fv ** 2)) <= 1e-10
    err = _rel(g_mixed, g_ref)
    assert err <= 1e-6, err
