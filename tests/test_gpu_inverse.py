"""Multi-resolution inversion of beta on the adjoint path.

1. The finest-level objective's gradient (forward and adjoint solved to
   1e-11, exact-boundary gradient, chain-rule-consistent regulariser, smooth
   Huber misfit) agrees with central differences in log(beta) to 1e-4
   relative on 3 seeded directions.
2. A twin experiment: beta_true = beta0 * exp(0.3 * smooth field); u_obs from
   a converged forward solve with beta_true; starting from beta0, the
   coarse-to-fine L-BFGS-B run (25 iterations per level, Tikhonov weight
   1e-2) cuts the finest-level misfit to <= 50 % of its starting value
   (measured 33 %; the Huber misfit with eps = 10 cannot fall below 6.3) and
   brings log(beta) closer to the truth where ice thicker than 100 m
   constrains it (measured error 12.2 -> 8.6; thinner cells carry little
   information about beta).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _physics(c, **kw):
    from glide_b200 import IcePhysics, SolverSettings
    ph = IcePhysics(c.ny, c.nx, c.dx, n_levels=c.n_levels, thklim=c.thklim, precision="fp64",
                    settings=SolverSettings(shift=0.0, err_threshold=1e-7), use_graphs=False, **kw)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    return ph


def _observe(ph, c, beta):
    ph.set_parameters(beta=beta)
    ph.reset_solution()
    ph.forward(c.dt, tol=1e-11, update_geometry=False)
    u, v = ph.grid.u.clone(), ph.grid.v.clone()
    ph.set_parameters(beta=c.beta)
    return u, v


def test_level_objective_gradient_matches_finite_differences():
    from glide_b200.inverse import LevelObjective, observation_hierarchy
    from glide_b200.synthetic import dome_case
    c = dome_case(0, n=32, dx=10000.0, n_levels=3)
    ph = _physics(c, gl_derivatives=True)
    u_obs, v_obs = _observe(ph, c, c.beta * 1.3)
    obs = observation_hierarchy(ph, u_obs, v_obs)
    obj = LevelObjective(ph, 0, obs[0][0], obs[0][1], c.dt, reg_weight=1e-2, loss="huber", tol=1e-11,
                         adj_tol=1e-11, exact=True, consistent_reg=True)
    x = np.log(c.beta).ravel()
    _, g = obj(x)
    rng = np.random.default_rng(11)
    eps = 1e-6
    for k in range(3):
        d = rng.standard_normal(x.size)
        fp, _ = obj(x + eps * d)
        fm, _ = obj(x - eps * d)
        fd = (fp - fm) / (2 * eps)
        ad = float(g @ d)
        assert abs(fd - ad) <= 1e-4 * abs(fd), (k, fd, ad)


def test_multiresolution_inversion_reduces_misfit():
    from glide_b200.inverse import invert_beta
    from glide_b200.synthetic import dome_case
    c = dome_case(2, n=64, dx=5000.0, n_levels=3)
    rng = np.random.default_rng(5)
    field = rng.standard_normal((8, 8))
    smooth = np.kron(field, np.ones((8, 8)))
    smooth = 0.25 * (np.roll(smooth, 1, 0) + np.roll(smooth, -1, 0) + np.roll(smooth, 1, 1) + np.roll(smooth, -1, 1))
    beta_true = c.beta * np.exp(0.3 * smooth)
    ph = _physics(c)
    u_obs, v_obs = _observe(ph, c, beta_true)
    beta, records = invert_beta(ph, u_obs, v_obs, c.dt, reg_weight=1e-2, loss="huber", maxiter=25,
                                consistent_reg=True, n_vcycles=8, n_adjoint_vcycles=4)
    fine = records[-1]
    assert fine["level"] == 0 and len(records) == 3
    assert fine["final_misfit"] <= 0.5 * fine["initial"]["misfit"], records
    ice = c.thickness > 100.0
    err0 = np.linalg.norm((np.log(c.beta) - np.log(beta_true))[ice])
    err1 = np.linalg.norm((np.log(beta.cpu().numpy()) - np.log(beta_true))[ice])
    assert err1 < 0.85 * err0, (err0, err1)


def test_time_stepped_objective_gradient_and_lbfgs():
    """The time-stepped inversion objective (4 steps, checkpoint every 2,
    noise-weighted chi^2 misfit per observation, Tikhonov 1e-3 on log beta):
    along directions where central differences at eps and 2 eps agree (the
    step map is smooth there), the gradient with a 1e-6 m adjoint active-set
    band agrees with them to 1e-4 relative; a few L-BFGS-B iterations lower
    the objective and record it per iteration."""
    from glide_b200.adjoint import time_stepped
    from glide_b200.inverse import TimeSteppedObjective, finite_difference_check, invert_time_stepped
    from glide_b200.synthetic import dome_case
    c = dome_case(0, n=32, dx=10000.0, n_levels=3)
    ph = _physics(c, gl_derivatives=True)
    H0 = torch.as_tensor(c.thickness, device="cuda")
    beta_true = torch.as_tensor(c.beta, device="cuda") * 1.5
    with torch.no_grad():
        u, v, _ = time_stepped(beta_true, H0, ph, c.dt, 4, 2, 1e-11, 1e-11)
    sig_u, sig_v = 0.02 * u.abs() + 1.0, 0.02 * v.abs() + 1.0
    obj = TimeSteppedObjective(ph, H0, u, v, c.dt, 4, 2, reg_weight=1e-3, tol=1e-11, adj_tol=1e-11,
                               sigma_u=sig_u, sigma_v=sig_v, normalize=True)
    x0 = np.log(c.beta).ravel()
    ph.settings.adj_active_tol = 1e-6
    f0, g = obj(x0)
    ph.settings.adj_active_tol = 0.1
    errs, pairs, smooth = finite_difference_check(obj, x0, n_directions=4, eps=1e-6, grads=[g], smooth_dirs=4)
    checked = [e for e, s in zip(errs[0], smooth) if s <= 1e-4]
    assert len(checked) >= 2, (smooth, errs)
    assert max(checked) <= 1e-4, (errs, smooth, pairs)
    x, rec = invert_time_stepped(obj, x0, maxiter=4)
    assert rec["final_total"] < f0
    assert len(rec["misfit_total_per_iteration"]) == rec["iterations"]
