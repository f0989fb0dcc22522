"""The hand-written VJP behind torch.autograd vs finite differences.

Loss L = 1/2 |u - u_obs|^2 + 1/2 |v - v_obs|^2 with u_obs from a perturbed
beta.  FP64, gl_derivatives on (so the JVP/VJP are the exact Jacobian),
exact-boundary gradient, forward and adjoint solved to 1e-11.
Central differences with eps = 1e-6 (relative to beta) on 16 seeded
directions must agree with the adjoint directional derivative to 1e-5
relative (the limit set by the solve tolerance over eps).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _setup(n=32, seed=0):
    from glide_b200 import IcePhysics, SolverSettings
    from glide_b200.synthetic import dome_case
    c = dome_case(seed, n=n, dx=5000.0 * 64 / n, n_levels=3)
    ph = IcePhysics(n, n, c.dx, n_levels=3, thklim=c.thklim, precision="fp64", gl_derivatives=True,
                    settings=SolverSettings(shift=0.0, err_threshold=1e-7), use_graphs=False)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    beta = torch.as_tensor(c.beta, device="cuda")
    H0 = torch.as_tensor(c.thickness, device="cuda")
    return c, ph, beta, H0


def _loss_fn(ph, H0, dt, u_obs, v_obs):
    from glide_b200.adjoint import ssa_step

    def L(beta):
        u, v, H = ssa_step(beta, H0, ph, dt, tol=TOL, adj_tol=TOL)
        return 0.5 * ((u - u_obs) ** 2).sum() + 0.5 * ((v - v_obs) ** 2).sum()
    return L


def test_step_gradient_matches_finite_differences():
    from glide_b200.adjoint import ssa_step
    c, ph, beta, H0 = _setup()
    with torch.no_grad():
        u_obs, v_obs, _ = ssa_step(beta * 1.3, H0, ph, c.dt, tol=TOL)
        u_obs, v_obs = u_obs.clone(), v_obs.clone()
    L = _loss_fn(ph, H0, c.dt, u_obs, v_obs)
    b = beta.clone().requires_grad_(True)
    loss = L(b)
    loss.backward()
    g = b.grad.clone()
    rng = np.random.default_rng(16)
    eps = 1e-6
    errs = []
    for k in range(16):
        d = torch.as_tensor(rng.standard_normal(beta.shape), device="cuda") * beta
        with torch.no_grad():
            fd = (L(beta + eps * d) - L(beta - eps * d)) / (2 * eps)
        ad = (g * d).sum()
        errs.append(abs(float(fd - ad)) / max(abs(float(fd)), 1e-30))
    assert max(errs) <= 1e-5, errs


def test_gradcheck_fast_mode():
    """torch.autograd.gradcheck (random-projection mode) on the step function."""
    from glide_b200.adjoint import ssa_step
    c, ph, beta, H0 = _setup(n=16)
    u_obs = torch.zeros(16, 17, dtype=torch.float64, device="cuda")
    v_obs = torch.zeros(17, 16, dtype=torch.float64, device="cuda")

    def f(b, h):
        u, v, H = ssa_step(b, h, ph, c.dt, tol=TOL, adj_tol=TOL)
        return 0.5 * ((u - u_obs) ** 2).sum() + 0.5 * ((v - v_obs) ** 2).sum()

    b = beta.clone().requires_grad_(True)
    h = H0.clone().requires_grad_(True)
    assert torch.autograd.gradcheck(f, (b, h), eps=1e-6, atol=1e-6, rtol=1e-4, fast_mode=True)


def test_time_stepped_checkpointed_gradient():
    """4 steps: the gradient w.r.t. beta is identical for checkpoint spacings
    1, 2 and 4 (recomputation replays the same solves), and agrees with
    central differences to 1e-4 relative on 3 seeded directions.

    The differences are taken where the step map is smooth: central
    differences at eps and 2*eps must agree first.  (The dome of seed 1 at
    dt = 10 a has a bistable margin cell, index (26, 7): a 1e-6 relative
    change of beta moves its thickness by ~150 m onto another solution
    branch; the FP64 NumPy oracle finds the same two branches.)"""
    from glide_b200.adjoint import time_stepped
    c, ph, beta, H0 = _setup(n=32, seed=0)

    def L(b, every=2):
        u, v, H = time_stepped(b, H0, ph, c.dt, n_steps=4, checkpoint_every=every, tol=TOL, adj_tol=TOL)
        return 0.5 * (u ** 2).sum() + 0.5 * (v ** 2).sum() + 1e-3 * (H ** 2).sum()

    grads = []
    for every in (2, 1, 4):
        b = beta.clone().requires_grad_(True)
        L(b, every).backward()
        grads.append(b.grad.clone())
    for other in grads[1:]:
        assert torch.equal(other, grads[0])
    g = grads[0]
    rng = np.random.default_rng(4)
    for k in range(3):
        d = torch.as_tensor(rng.standard_normal(beta.shape), device="cuda") * beta
        with torch.no_grad():
            fd = ((L(beta + 1e-6 * d) - L(beta - 1e-6 * d)) / 2e-6).item()
            fd2 = ((L(beta + 2e-6 * d) - L(beta - 2e-6 * d)) / 4e-6).item()
        assert abs(fd2 - fd) <= 1e-4 * abs(fd), "finite differences cross a solution branch"
        ad = (g * d).sum().item()
        assert abs(fd - ad) <= 1e-4 * abs(fd), (k, fd, ad)


def test_adjoint_recovers_from_a_diverging_cycle():
    """Mixed precision adjoint to a tolerance by cycles and sweeps
    (``adjoint_krylov=0``): a cycle that leaves the multiplier non-finite
    (planted on the host by overwriting it with NaN after the second cycle)
    is undone, the fine-level sweeps finish from the best multiplier, and the
    gradient equals the undisturbed solve's (FGMRES) to the tolerance's
    accuracy."""
    from glide_b200 import IcePhysics, SolverSettings
    from glide_b200.synthetic import dome_case
    c = dome_case(0, n=64, dx=5000.0, n_levels=3)

    def physics(krylov=30):
        ph = IcePhysics(64, 64, c.dx, n_levels=3, thklim=c.thklim, precision="mixed",
                        settings=SolverSettings(shift=0.0, err_threshold=1e-7), adjoint_krylov=krylov)
        ph.set_geometry(c.bed, c.thickness)
        ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
        ph.forward(c.dt, tol=1e-9, update_geometry=False)
        return ph

    gen = torch.Generator().manual_seed(5)
    ref = physics()
    cu = torch.randn(tuple(ref.grid.u.shape), generator=gen, dtype=torch.float64).cuda()
    cv = torch.randn(tuple(ref.grid.v.shape), generator=gen, dtype=torch.float64).cuda()
    cH = torch.zeros_like(ref.grid.H)
    g_ref = ref.adjoint(cu, cv, cH, tol=1e-8).clone()
    assert ref.last_adjoint_info["rel_residual"] <= 1e-8

    ph = physics(krylov=0)   # the cycles-then-sweeps solve
    step = ph._adjoint_dc_step
    calls = []

    def planted(cfg):
        step(cfg)
        calls.append(1)
        if len(calls) == 2:
            ph.grid.Lambda.fill_(float("nan"))
    ph._adjoint_dc_step = planted
    g = ph.adjoint(cu, cv, cH, tol=1e-8)
    info = ph.last_adjoint_info
    assert info.get("cycle_restored"), info
    assert info["rel_residual"] <= 1e-8, info
    assert torch.isfinite(g).all()
    assert float((g - g_ref).norm() / g_ref.norm()) <= 1e-6
