"""Multi-resolution inversion of basal friction on the adjoint path.

Restates the coarse-to-fine driver of examples/antarctica/antarctica_inverse.py:
148-289 on this package: observations are restricted to every multigrid level
(:128-138); from the coarsest level to the finest, L-BFGS-B (scipy's
``fmin_l_bfgs_b``, bounds (-6, 5) on log(beta), ``factr`` 1e10, ``m`` 15)
minimises misfit + ``reg_weight`` * Tikhonov(beta) over log(beta); the optimum
is prolongated (bilinear, glide/kernels.py:216-236) as the next level's start.

One objective evaluation at level k (antarctica_inverse.py:174-241):
beta = exp(x); u = v = 0, H = H_prev; restrict the parameters below k;
f_H = H_prev/dt + smb; forward V-cycles on the sub-hierarchy from k; misfit and
its gradient; f_adj = -dL/d(u, v), Lambda = 0; adjoint V-cycles; grad_beta;
d/d(log beta) = beta * grad_beta; plus the regulariser.

Two switches go beyond the reference:

* ``tol`` / ``adj_tol`` on the finest level solve forward and adjoint to a
  relative residual with ``IcePhysics.forward``/``adjoint`` (the reference runs
  5 forward and 2 adjoint V-cycles, so its gradient is the adjoint of an
  unconverged state);
* ``consistent_reg``: the reference adds the Tikhonov gradient taken with
  respect to beta to the gradient with respect to log(beta)
  (antarctica_inverse.py:230-235); with ``consistent_reg=True`` it is
  multiplied by beta first (the chain rule), so that the objective and its
  gradient agree.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .kernels import prolongate_cell_centered, restrict_hfacet, restrict_vfacet
from .losses import KINDS, misfit, tikhonov
from .solver import adjoint_vcycle, fascd_vcycle, restrict_parameters_to_hierarchy


def observation_hierarchy(physics, u_obs, v_obs):
    """(u_obs, v_obs) on every level, finest first (antarctica_inverse.py:128-133)."""
    g = physics.grid
    u = torch.as_tensor(u_obs, dtype=g.dtype, device=g.device)
    v = torch.as_tensor(v_obs, dtype=g.dtype, device=g.device)
    out = [(u, v)]
    while g.child is not None:
        u, v = restrict_vfacet(u), restrict_hfacet(v)
        out.append((u, v))
        g = g.child
    return out


class LevelObjective:
    """Misfit + regulariser and its gradient in log(beta) at one level."""

    def __init__(self, physics, level, u_obs, v_obs, dt, *, reg_weight=1e-4, loss="abs", n_vcycles=5,
                 n_adjoint_vcycles=2, tol=None, adj_tol=None, exact=False, consistent_reg=False):
        if physics.precision == "mixed":
            raise ValueError("the inversion runs on the fp32 or fp64 hierarchy")
        self.ph = physics
        self.level = int(level)
        self.grid = physics.grids[self.level]
        self.u_obs, self.v_obs = u_obs, v_obs
        self.dt = float(dt)
        self.reg_weight = float(reg_weight)
        if loss not in KINDS:
            raise ValueError(f"loss must be one of {sorted(KINDS)}")
        self.loss = loss
        self.n_vcycles, self.n_adjoint = int(n_vcycles), int(n_adjoint_vcycles)
        self.tol, self.adj_tol, self.exact = tol, adj_tol, bool(exact)
        self.consistent_reg = bool(consistent_reg)
        self.evaluations = 0
        self.last = {}

    def _forward(self, g):
        ph = self.ph
        if self.level == 0 and self.tol is not None:
            ph.reset_solution()
            ph.forward(self.dt, tol=self.tol, update_geometry=False)
            return
        g.u.zero_()
        g.v.zero_()
        g.H.copy_(g.H_prev)
        restrict_parameters_to_hierarchy(g)
        g.f_H.copy_(g.H_prev / g.dt + g.smb)
        for _ in range(self.n_vcycles):
            fascd_vcycle(g, ph.thklim, finest=True, settings=ph.settings)

    def _adjoint(self, g, du, dv):
        ph = self.ph
        if self.level == 0 and self.adj_tol is not None:
            return ph.adjoint(du, dv, torch.zeros_like(g.H), tol=self.adj_tol, exact=self.exact)
        g.f_adj_u.copy_(-du)
        g.f_adj_v.copy_(-dv)
        g.f_adj_H.zero_()
        g.Lambda.zero_()
        saved = ph.settings.exact_adjoint
        ph.settings.exact_adjoint = self.exact
        try:
            for _ in range(self.n_adjoint):
                adjoint_vcycle(g, ph.settings, ph.thklim)
        finally:
            ph.settings.exact_adjoint = saved
        return g.compute_grad_beta(exact_boundary=self.exact)

    def __call__(self, x):
        """(objective, gradient) for L-BFGS-B; x = log(beta) as float64, flattened."""
        g = self.grid
        for lv in self.ph.grids[self.level:]:
            lv.dt = self.dt
        self.ph._set_dt(self.dt)
        log_beta = torch.as_tensor(np.asarray(x, dtype=np.float64).reshape(g.ny, g.nx), device=g.device)
        g.beta.copy_(torch.exp(log_beta).to(g.dtype))
        self._forward(g)
        J_dev, du, dv = misfit(g.u, g.v, self.u_obs, self.v_obs, kind=self.loss)   # fused loss + gradient
        grad_beta = self._adjoint(g, du, dv)
        grad = g.beta * grad_beta
        tik_dev, tik_grad = tikhonov(g.beta)
        J, tik = float(J_dev), float(tik_dev)
        if self.consistent_reg:
            tik_grad = tik_grad * g.beta
        total = J + self.reg_weight * tik
        grad = grad + self.reg_weight * tik_grad
        self.evaluations += 1
        self.last = {"misfit": J, "reg": self.reg_weight * tik, "total": total}
        return total, grad.double().cpu().numpy().ravel()


def invert_beta(physics, u_obs, v_obs, dt, *, reg_weight=1e-4, loss="abs", bounds=(-6.0, 5.0), factr=1e10, m=15,
                maxiter=15000, levels=None, n_vcycles=5, n_adjoint_vcycles=2, tol=None, adj_tol=None, exact=False,
                consistent_reg=False, callback=None):
    """Coarse-to-fine L-BFGS-B over log(beta) (antarctica_inverse.py:148-289).

    ``physics`` carries the geometry, B, smb and the starting beta.  ``levels``
    lists the level indices to optimise, coarsest first (default: all).
    Returns the finest optimised beta (a tensor, also left in physics.grid.beta)
    and one record per level (objective evaluations, final misfit, scipy info).
    """
    from scipy.optimize import fmin_l_bfgs_b

    obs = observation_hierarchy(physics, u_obs, v_obs)
    grids = physics.grids
    order = list(range(len(grids) - 1, -1, -1)) if levels is None else list(levels)
    # the starting beta of the coarsest optimised level comes from the finest one
    restrict_parameters_to_hierarchy(physics.grid)
    records = []
    for pos, k in enumerate(order):
        g = grids[k]
        obj = LevelObjective(physics, k, obs[k][0], obs[k][1], dt, reg_weight=reg_weight, loss=loss,
                             n_vcycles=n_vcycles, n_adjoint_vcycles=n_adjoint_vcycles,
                             tol=tol if k == 0 else None, adj_tol=adj_tol if k == 0 else None, exact=exact,
                             consistent_reg=consistent_reg)
        x0 = torch.log(g.beta).double().cpu().numpy().ravel()
        f0, _ = obj(x0)
        first = dict(obj.last)
        cb = (lambda xk, _k=k: callback(_k, xk)) if callback is not None else None
        x, f, info = fmin_l_bfgs_b(obj, x0, bounds=[bounds] * x0.size, factr=factr, m=m, maxiter=maxiter,
                                   callback=cb)
        g.beta.copy_(torch.exp(torch.as_tensor(x.reshape(g.ny, g.nx), device=g.device)).to(g.dtype))
        g.mask.zero_()
        records.append({"level": k, "shape": (g.ny, g.nx), "evaluations": obj.evaluations, "initial": first,
                        "final_total": float(f), "final_misfit": obj.last.get("misfit", math.nan),
                        "warnflag": int(info["warnflag"]), "iterations": int(info["nit"])})
        if pos + 1 < len(order) and order[pos + 1] == k - 1:
            prolongate_cell_centered(g.beta, H_fine=grids[k - 1].beta)
    return physics.grid.beta, records


# ---------------------------------------------------------------------------
# time-stepped inversion (no counterpart in the reference, whose adjoint is
# single-step, glide/physics.py:211-242)
# ---------------------------------------------------------------------------
class TimeSteppedObjective:
    """L(log beta) = 1/2 |u_n - u_obs|^2 + 1/2 |v_n - v_obs|^2 + reg_weight * T(log beta)
    after ``n_steps`` implicit steps from H0, and its gradient in log beta.

    The steps run through ``glide_b200.adjoint.TimeStepper`` (checkpoints every
    ``checkpoint_every`` steps, segments recomputed in the backward pass); the
    misfit gradient is beta * dL/dbeta from the hand-written adjoint, the
    Tikhonov term (``losses.tikhonov``) is taken in log beta directly.
    ``x`` is the flattened log beta (float64 NumPy), as scipy's L-BFGS-B
    passes it."""

    def __init__(self, physics, H0, u_obs, v_obs, dt, n_steps, checkpoint_every=10, reg_weight=1e-3, tol=1e-8,
                 adj_tol=1e-8, max_vcycles=60, sigma_u=None, sigma_v=None, normalize=False):
        g = physics.grid
        self.ph, self.dt, self.n, self.every = physics, float(dt), int(n_steps), int(checkpoint_every)
        self.H0 = torch.as_tensor(H0, dtype=g.dtype, device=g.device)
        self.u_obs = torch.as_tensor(u_obs, dtype=g.dtype, device=g.device)
        self.v_obs = torch.as_tensor(v_obs, dtype=g.dtype, device=g.device)
        # misfit weights 1/sigma^2 (1 without sigma), divided by the number of observations with ``normalize``
        scale = 1.0 / (self.u_obs.numel() + self.v_obs.numel()) if normalize else 1.0
        self.w_u = scale / torch.as_tensor(sigma_u, dtype=g.dtype, device=g.device) ** 2 if sigma_u is not None \
            else torch.full_like(self.u_obs, scale)
        self.w_v = scale / torch.as_tensor(sigma_v, dtype=g.dtype, device=g.device) ** 2 if sigma_v is not None \
            else torch.full_like(self.v_obs, scale)
        self.reg_weight, self.tol, self.adj_tol, self.max_vcycles = float(reg_weight), tol, adj_tol, max_vcycles
        self.shape = (g.ny, g.nx)
        self.evaluations = 0
        self.max_step_rel = 0.0   # largest |r|/|r0| any step of any evaluation reached
        self.last = {}

    def value_and_grad(self, logb):
        """Objective and gradient for a log-beta tensor (device, working dtype)."""
        from .adjoint import time_stepped
        beta = torch.exp(logb.detach()).requires_grad_(True)
        self.ph.solve_log = []
        u, v, _ = time_stepped(beta, self.H0, self.ph, self.dt, self.n, self.every, self.tol, self.adj_tol,
                               self.max_vcycles)
        J = self._misfit(u, v)
        J.backward()
        t, gt = tikhonov(logb.detach())
        grad = beta.grad * beta.detach() + self.reg_weight * gt
        total = float(J.detach()) + self.reg_weight * float(t)
        self.evaluations += 1
        rels = [r for r in self.ph.solve_log if r is not None]
        self.ph.solve_log = None
        self.last = {"misfit": float(J.detach()), "reg": self.reg_weight * float(t), "total": total,
                     "max_step_rel_residual": max(rels) if rels else None,
                     "adjoint_rel_residual": getattr(self.ph, "last_adjoint_info", {}).get("rel_residual")}
        self.max_step_rel = max(self.max_step_rel, max(rels) if rels else 0.0)
        return total, grad

    def _misfit(self, u, v):
        return 0.5 * (self.w_u * (u - self.u_obs) ** 2).sum() + 0.5 * (self.w_v * (v - self.v_obs) ** 2).sum()

    def _logb(self, x):
        g = self.ph.grid
        return torch.as_tensor(np.asarray(x).reshape(self.shape), dtype=g.dtype, device=g.device)

    def __call__(self, x):
        total, grad = self.value_and_grad(self._logb(x))
        return total, grad.double().cpu().numpy().ravel()

    def value(self, x):
        """The objective alone (forward steps only, no adjoint)."""
        from .adjoint import time_stepped
        logb = self._logb(x)
        self.ph.solve_log = []
        with torch.no_grad():
            u, v, _ = time_stepped(torch.exp(logb), self.H0, self.ph, self.dt, self.n, self.every, self.tol,
                                   self.adj_tol, self.max_vcycles)
            J = self._misfit(u, v)
        rels = [r for r in self.ph.solve_log if r is not None]
        self.ph.solve_log = None
        self.max_step_rel = max(self.max_step_rel, max(rels) if rels else 0.0)
        t, _ = tikhonov(logb)
        return float(J) + self.reg_weight * float(t)


def finite_difference_check(objective, x, n_directions=16, eps=1e-6, seed=0, grads=None, smooth_dirs=0):
    """Central differences (L(x + eps d) - L(x - eps d)) / (2 eps) of a
    ``TimeSteppedObjective`` along ``n_directions`` seeded unit-variance
    directions d, against grad . d from its adjoint (or, with ``grads``, from
    each of several precomputed gradients).  Returns the relative differences
    |fd - ad| / |fd| (a list per gradient when ``grads`` is given), the pairs
    (fd, ad) and, for the first ``smooth_dirs`` directions, the relative
    difference of the central differences at eps and 2 eps: a large one means
    the step map is not smooth along d at this scale (a cell changes solution
    branch), so no gradient can match that direction's differences."""
    rng = np.random.default_rng(seed)
    if grads is None:
        _, grad = objective(x)
        glist = [grad]
    else:
        glist = list(grads)
    errs = [[] for _ in glist]
    pairs, smooth = [], []
    for k in range(n_directions):
        d = rng.standard_normal(x.size)
        fp = objective.value(x + eps * d)
        fm = objective.value(x - eps * d)
        fd = (fp - fm) / (2.0 * eps)
        ads = [float(g @ d) for g in glist]
        for e, ad in zip(errs, ads):
            e.append(abs(fd - ad) / max(abs(fd), 1e-300))
        pairs.append((fd, *ads))
        if k < smooth_dirs:
            fd2 = (objective.value(x + 2 * eps * d) - objective.value(x - 2 * eps * d)) / (4.0 * eps)
            smooth.append(abs(fd2 - fd) / max(abs(fd), 1e-300))
    return (errs[0] if grads is None else errs), pairs, smooth


def invert_time_stepped(objective, x0, *, maxiter=200, bounds=(-6.0, 5.0), m=15, factr=1e7, callback=None,
                        max_seconds=None):
    """L-BFGS-B over log beta of a ``TimeSteppedObjective`` (``maxiter``
    iterations at most; with ``max_seconds``, no new iteration starts after
    that wall time).  Returns the last accepted iterate and a record (with the
    misfit and objective after every iteration)."""
    import time

    from scipy.optimize import minimize
    t0 = time.time()
    f0, _ = objective(x0)
    first = dict(objective.last)
    history = []
    best = {"x": np.array(x0, dtype=np.float64), "f": f0}
    stopped = {"time": False}

    def cb(xk):
        history.append((objective.last["misfit"], objective.last["total"]))
        best["x"] = np.array(xk, dtype=np.float64)
        best["f"] = objective.last["total"]
        if callback is not None:
            callback(xk)
        if max_seconds is not None and time.time() - t0 > max_seconds:
            stopped["time"] = True
            raise StopIteration
    res = minimize(objective, x0, jac=True, method="L-BFGS-B", bounds=[bounds] * x0.size, callback=cb,
                   options={"maxiter": maxiter, "maxcor": m, "ftol": factr * np.finfo(float).eps})
    x = res.x if not stopped["time"] else best["x"]
    return x, {"initial": first, "final": dict(objective.last), "final_total": float(best["f"]),
               "iterations": len(history), "evaluations": objective.evaluations,
               "stopped_on_time": stopped["time"], "message": str(res.message),
               "misfit_total_per_iteration": history}
