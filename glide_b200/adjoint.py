"""Differentiable forward steps: the hand-written adjoint behind autograd.

``ssa_step(beta, H_prev, physics, dt)`` solves one implicit step and returns
(u, v, H) as tensors that carry gradients back to ``beta`` and ``H_prev``.
Its backward is the adjoint of the converged step, solved with the adjoint
V-cycle (glide/solver.py:160-220) on the kernels of this package:

    J(U)^T lam = -(dL/du, dL/dv, dL/dH)            (J: Jacobian of F(U) - f)
    dL/dbeta   = lam^T dF/dbeta                       (glide_grad_beta, exact)
    dL/dH_prev = lam_H^T dF_H/dH_prev = -(1 - m) lam_H / dt

The last term follows from f_H = H_prev/dt + smb (glide/physics.py:173); it
is new here (the reference adjoint returns grad_beta only).  Rows of cells
held at the thickness limit (mask m: H <= gamma + 0.1 by default,
``SolverSettings.adj_active_tol``; glide/grid.py:332)
are identity rows of J, so they pass no sensitivity to H_prev.

``TimeStepper`` chains n steps; its backward recomputes each segment of
``checkpoint_every`` steps once from a stored thickness (the only state
carried between steps), keeps the segment's solved states, and runs the
adjoint steps of that segment in reverse at those states.
"""
from __future__ import annotations

import torch


def _solve(physics, beta, H_prev, dt, tol, max_vcycles):
    g = physics.grid
    physics.set_parameters(beta=beta)
    g.H_prev.copy_(H_prev)
    g.H.copy_(H_prev)
    if physics.grid32 is not None:
        physics.grid32.H_prev.copy_(H_prev)
    g.u.zero_()
    g.v.zero_()
    physics.forward(dt, tol=tol, max_vcycles=max_vcycles, update_geometry=False, max_finish_sweeps=20000)
    log = getattr(physics, "solve_log", None)
    if isinstance(log, list):   # relative residual each solve reached (diagnostics of callers)
        log.append(physics.last_info.get("rel_residual"))
    return g.u.clone(), g.v.clone(), g.H.clone()


def _restore(physics, beta, H_prev, U, dt):
    """Put a solved step back as the linearisation point of its adjoint
    (parameters, H_prev, dt and the converged state) without solving again.
    The coarse levels, where the adjoint V-cycle linearises its coarse
    corrections, get the restricted state, so the adjoint depends on the
    step's state alone (not on which solve ran last)."""
    from .kernels import restrict_cell_centered, restrict_hfacet, restrict_vfacet
    g = physics.grid
    physics.set_parameters(beta=beta)
    physics._set_dt(dt)
    g.H_prev.copy_(H_prev)
    if physics.grid32 is not None:
        physics.grid32.H_prev.copy_(H_prev)
        physics.grid32.U.copy_(U)
        hier = physics.grids32
    else:
        hier = physics.grids
    g.U.copy_(U)
    g.f_H.copy_(g.H_prev / dt + g.smb)
    for par, ch in zip(hier[:-1], hier[1:]):
        restrict_vfacet(par.u, u_coarse=ch.u)
        restrict_hfacet(par.v, v_coarse=ch.v)
        restrict_cell_centered(par.H, f_coarse=ch.H)


def _adjoint(physics, du, dv, dH, dt, adj_tol, max_vcycles):
    g = physics.grid
    grad_beta = physics.adjoint(du, dv, dH, tol=adj_tol, max_vcycles=max_vcycles, exact=True)
    g.compute_mask(physics.settings.adj_active_tol)
    grad_Hprev = -(1.0 - g.mask) * g.lambda_H / dt
    g.mask.zero_()
    return grad_beta.clone(), grad_Hprev.clone()


class SSAStep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, beta, H_prev, physics, dt, tol, adj_tol, max_vcycles):
        u, v, H = _solve(physics, beta.detach(), H_prev.detach(), dt, tol, max_vcycles)
        ctx.physics, ctx.dt, ctx.adj_tol, ctx.max_vcycles, ctx.tol = physics, dt, adj_tol, max_vcycles, tol
        ctx.save_for_backward(beta.detach(), H_prev.detach(), u, v, H)
        return u, v, H

    @staticmethod
    def backward(ctx, gu, gv, gH):
        beta, H_prev, u, v, H = ctx.saved_tensors
        ph = ctx.physics
        g = ph.grid
        # restore the linearisation point (another step may have used the solver)
        if not (torch.equal(g.u, u) and torch.equal(g.v, v) and torch.equal(g.H, H)):
            _solve(ph, beta, H_prev, ctx.dt, ctx.tol, ctx.max_vcycles)
        z = lambda t, like: torch.zeros_like(like) if t is None else t
        gb, gh = _adjoint(ph, z(gu, u), z(gv, v), z(gH, H), ctx.dt, ctx.adj_tol, ctx.max_vcycles)
        return gb.to(beta.dtype), gh.to(H_prev.dtype), None, None, None, None, None


def ssa_step(beta, H_prev, physics, dt, tol=1e-10, adj_tol=1e-10, max_vcycles=60):
    """One differentiable implicit step; returns (u, v, H)."""
    return SSAStep.apply(beta, H_prev, physics, dt, tol, adj_tol, max_vcycles)


class TimeStepper(torch.autograd.Function):
    """n implicit steps from H0 with fixed beta; returns the final (u, v, H).

    Memory: one thickness per checkpoint (every ``checkpoint_every`` steps);
    the backward recomputes the steps of a segment from its checkpoint and
    runs their adjoints in reverse order."""

    @staticmethod
    def forward(ctx, beta, H0, physics, dt, n_steps, checkpoint_every, tol, adj_tol, max_vcycles):
        beta = beta.detach()
        H = H0.detach().clone()
        checkpoints = {0: H.clone()}
        u = v = None
        for k in range(n_steps):
            u, v, H = _solve(physics, beta, H, dt, tol, max_vcycles)
            if (k + 1) % checkpoint_every == 0 and k + 1 < n_steps:
                checkpoints[k + 1] = H.clone()
        ctx.physics, ctx.dt, ctx.n, ctx.every = physics, dt, n_steps, checkpoint_every
        ctx.tol, ctx.adj_tol, ctx.max_vcycles = tol, adj_tol, max_vcycles
        ctx.checkpoints = checkpoints
        ctx.save_for_backward(beta)
        return u, v, H

    @staticmethod
    def backward(ctx, gu, gv, gH):
        (beta,) = ctx.saved_tensors
        ph, dt = ctx.physics, ctx.dt
        n, every = ctx.n, ctx.every
        grad_beta = torch.zeros_like(beta)
        # sensitivities carried backwards: w.r.t. the final u, v, H first
        cu, cv, cH = gu, gv, gH
        starts = sorted(ctx.checkpoints)
        for s0 in reversed(starts):
            s1 = min(s0 + every, n)
            # recompute the segment once, keeping each step's starting thickness and solved state
            steps = []
            H_in = ctx.checkpoints[s0]
            for k in range(s0, s1):
                u, v, H = _solve(ph, beta, H_in, dt, ctx.tol, ctx.max_vcycles)
                steps.append((H_in, ph.grid.U.detach().clone()))
                H_in = H
            for k in range(s1 - 1, s0 - 1, -1):
                H_in, U = steps[k - s0]
                _restore(ph, beta, H_in, U, dt)
                u, v, H = ph.grid.u, ph.grid.v, ph.grid.H
                z = lambda t, like: torch.zeros_like(like) if t is None else t
                gb, gh = _adjoint(ph, z(cu, u), z(cv, v), z(cH, H), dt, ctx.adj_tol, ctx.max_vcycles)
                grad_beta += gb.to(grad_beta.dtype)
                # the previous step's outputs enter this step only through H_prev
                cu, cv, cH = None, None, gh
        return grad_beta, cH, None, None, None, None, None, None, None


def time_stepped(beta, H0, physics, dt, n_steps, checkpoint_every=10, tol=1e-10, adj_tol=1e-10, max_vcycles=60):
    return TimeStepper.apply(beta, H0, physics, dt, n_steps, checkpoint_every, tol, adj_tol, max_vcycles)
