"""FP64 NumPy restatement of GLIDE's transfers, FASCD and adjoint V-cycles.

Test infrastructure only (see ``oracle/ssa.py``).  Transfers restate
glide/cuda/utility.cu:1-337, the V-cycles restate glide/solver.py:71-220,
the level bookkeeping restates glide/grid.py, and ``OracleIcePhysics``
restates the IcePhysics API of glide/physics.py:49-242.
"""
from __future__ import annotations

import numpy as np

from . import ssa
from .ssa import Params
from .vanka import local_cell_on, vanka_adjoint_color, vanka_deltas


# ---------------------------------------------------------------------------
# transfers (glide/cuda/utility.cu)
# ---------------------------------------------------------------------------

def restrict_u(uf):
    """Tangential 2-average (utility.cu:1-19)."""
    return 0.5 * (uf[0::2, 0::2] + uf[1::2, 0::2])


def restrict_v(vf):
    """utility.cu:125-143."""
    return 0.5 * (vf[0::2, 0::2] + vf[0::2, 1::2])


def restrict_cell(hf):
    """4-cell average (utility.cu:56-75)."""
    return 0.25 * (hf[0::2, 0::2] + hf[0::2, 1::2] + hf[1::2, 0::2] + hf[1::2, 1::2])


def restrict_max_pool(hf):
    """utility.cu:77-101."""
    return np.maximum(np.maximum(hf[0::2, 0::2], hf[0::2, 1::2]), np.maximum(hf[1::2, 0::2], hf[1::2, 1::2]))


def prolong_cell_inject(hc):
    """utility.cu:104-123."""
    return np.repeat(np.repeat(hc, 2, axis=0), 2, axis=1)


def prolong_u_linear(uc):
    """Linear in x, constant in y (utility.cu:21-54)."""
    nyc, nxc1 = uc.shape
    nxc = nxc1 - 1
    uf = np.empty((2 * nyc, 2 * nxc + 1))
    rows = np.repeat(uc, 2, axis=0)
    uf[:, 0::2] = rows
    uf[:, 1::2] = 0.5 * (rows[:, :-1] + rows[:, 1:])
    return uf


def prolong_v_linear(vc):
    """utility.cu:145-178."""
    nyc1, nxc = vc.shape
    nyc = nyc1 - 1
    vf = np.empty((2 * nyc + 1, 2 * nxc))
    cols = np.repeat(vc, 2, axis=1)
    vf[0::2, :] = cols
    vf[1::2, :] = 0.5 * (cols[:-1, :] + cols[1:, :])
    return vf


def _bilinear(c, Jf, If, jmax, imax):
    Jf = np.clip(Jf, 0.0, float(jmax))
    If = np.clip(If, 0.0, float(imax))
    Jlo = Jf.astype(np.int64)
    Ilo = If.astype(np.int64)
    Jhi = np.minimum(Jlo + 1, jmax)
    Ihi = np.minimum(Ilo + 1, imax)
    ty = Jf - Jlo
    tx = If - Ilo
    v00 = c[Jlo, Ilo]; v01 = c[Jlo, Ihi]; v10 = c[Jhi, Ilo]; v11 = c[Jhi, Ihi]
    return (1.0 - ty) * ((1.0 - tx) * v00 + tx * v01) + ty * ((1.0 - tx) * v10 + tx * v11)


def prolong_u_bilinear(uc):
    """utility.cu:180-232."""
    nyc, nxc1 = uc.shape
    nxc = nxc1 - 1
    j = np.arange(2 * nyc)[:, None].astype(float)
    i = np.arange(2 * nxc + 1)[None, :].astype(float)
    return _bilinear(uc, np.broadcast_to((j - 0.5) * 0.5, (2 * nyc, 2 * nxc + 1)),
                     np.broadcast_to(i * 0.5, (2 * nyc, 2 * nxc + 1)), nyc - 1, nxc)


def prolong_v_bilinear(vc):
    """utility.cu:235-287."""
    nyc1, nxc = vc.shape
    nyc = nyc1 - 1
    j = np.arange(2 * nyc + 1)[:, None].astype(float)
    i = np.arange(2 * nxc)[None, :].astype(float)
    return _bilinear(vc, np.broadcast_to(j * 0.5, (2 * nyc + 1, 2 * nxc)),
                     np.broadcast_to((i - 0.5) * 0.5, (2 * nyc + 1, 2 * nxc)), nyc, nxc - 1)


def prolong_cell_bilinear(hc):
    """utility.cu:289-337."""
    nyc, nxc = hc.shape
    j = np.arange(2 * nyc)[:, None].astype(float)
    i = np.arange(2 * nxc)[None, :].astype(float)
    return _bilinear(hc, np.broadcast_to((j - 0.5) * 0.5, (2 * nyc, 2 * nxc)),
                     np.broadcast_to((i - 0.5) * 0.5, (2 * nyc, 2 * nxc)), nyc - 1, nxc - 1)


# ---------------------------------------------------------------------------
# level state (glide/grid.py)
# ---------------------------------------------------------------------------

class Level:
    """One multigrid level; attribute names follow glide/grid.py:79-158."""

    def __init__(self, ny, nx, dx, dt, p: Params):
        self.ny, self.nx, self.dx, self.dt, self.p = ny, nx, float(dx), float(dt), p
        self.child = None
        z = lambda *s: np.zeros(s)
        self.u, self.v, self.H = z(ny, nx + 1), z(ny + 1, nx), z(ny, nx)
        self.H_prev = z(ny, nx)
        self.f_u, self.f_v, self.f_H = z(ny, nx + 1), z(ny + 1, nx), z(ny, nx)
        self.w_u, self.w_v, self.w_H = z(ny, nx + 1), z(ny + 1, nx), z(ny, nx)
        self.y_u, self.y_v, self.y_H = z(ny, nx + 1), z(ny + 1, nx), z(ny, nx)
        self.lu, self.lv, self.lH = z(ny, nx + 1), z(ny + 1, nx), z(ny, nx)
        self.fa_u, self.fa_v, self.fa_H = z(ny, nx + 1), z(ny + 1, nx), z(ny, nx)
        self.chi, self.phi = z(ny, nx), z(ny, nx)
        self.bed, self.beta, self.B, self.smb = z(ny, nx), z(ny, nx), z(ny, nx), z(ny, nx)
        self.mask, self.error_mask, self.gamma = z(ny, nx), z(ny, nx), z(ny, nx)
        self.r_u = self.r_v = self.r_H = None
        self.shift = 1.0

    def spawn_child(self):
        """glide/grid.py:167-180: coarse levels keep n, eps_reg, water_drag and
        calving_rate but fall back to gl_sigmoid_c=0.1, gl_derivatives=False."""
        p = self.p
        cp_ = Params(n=p.n, eps_reg=p.eps_reg, water_drag=p.water_drag, calving_rate=p.calving_rate)
        self.child = Level(self.ny // 2, self.nx // 2, self.dx * 2, self.dt, cp_)
        return self.child

    # -- operators ---------------------------------------------------------
    def compute_residual(self, fischer_burmeister=False):
        self.r_u, self.r_v, self.r_H = ssa.residual(self.u, self.v, self.H, self.f_u, self.f_v, self.f_H,
                                                    self.bed, self.B, self.beta, self.mask, self.gamma,
                                                    self.p, self.dx, self.dt)
        if fischer_burmeister:
            a, b = self.r_H, self.H - self.gamma
            return a + b - np.sqrt(a * a + b * b)

    def compute_F(self):
        z = np.zeros_like
        return ssa.residual(self.u, self.v, self.H, z(self.f_u), z(self.f_v), z(self.f_H), self.bed, self.B,
                            self.beta, self.mask, self.gamma, self.p, self.dx, self.dt)

    def vjp(self):
        return ssa.vjp(self.u, self.v, self.H, self.lu, self.lv, self.lH, self.bed, self.B, self.beta, self.mask,
                       self.gamma, self.p, self.dx, self.dt)

    def vanka_sweep(self, n_iter, n_inner=10, omega=0.5, local=False):
        """glide/grid.py:305-317 (U += omega * delta after each launch)."""
        for _ in range(n_iter):
            on = local_cell_on(self.error_mask) if local else None
            if on is not None and not on.any():
                continue
            du, dv, dH = vanka_deltas(self.u, self.v, self.H, self.f_u, self.f_v, self.f_H, self.bed, self.B,
                                      self.beta, self.gamma, self.p, self.dx, self.dt, n_inner, on,
                                      shift=self.shift)
            self.u = self.u + omega * du
            self.v = self.v + omega * dv
            self.H = self.H + omega * dH

    def compute_mask(self, tol=1e-1):
        """glide/grid.py:332-334."""
        self.mask = (self.H <= (self.gamma + tol)).astype(float)

    def adjoint_residual(self):
        vu, vv, vH = self.vjp()
        return self.fa_u - vu, self.fa_v - vv, self.fa_H - vH

    def vanka_sweep_adjoint(self, n_iter, omega=0.5):
        """glide/grid.py:319-330: per colour, r_adj = f_adj - VJP(lambda) then solve."""
        for _ in range(n_iter):
            for color in (0, 1):
                r = self.adjoint_residual()
                self.lu, self.lv, self.lH = vanka_adjoint_color(
                    self.lu, self.lv, self.lH, self.mask, r, self.u, self.v, self.H, self.bed, self.B,
                    self.beta, self.gamma, self.p, self.dx, self.dt, color, omega)

    def compute_grad_beta(self, exact_boundary=False):
        """glide/grid.py:336-355."""
        return ssa.grad_beta(self.u, self.v, self.H, self.lu, self.lv, self.bed, self.beta, self.p,
                             exact_boundary=exact_boundary)


def restrict_parameters(g: Level):
    """glide/solver.py:53-61."""
    c = g.child
    c.bed = restrict_cell(g.bed); c.B = restrict_cell(g.B); c.beta = restrict_cell(g.beta)
    c.H_prev = restrict_cell(g.H_prev); c.smb = restrict_cell(g.smb)


def restrict_parameters_to_hierarchy(g: Level):
    """glide/solver.py:64-68."""
    while g.child is not None:
        restrict_parameters(g)
        g = g.child


def error_mask(g: Level, threshold=0.01):
    """Local error indicator of the post-smoothing loop (glide/solver.py:148-154)."""
    g.compute_residual()
    a = g.r_H
    b = g.H - g.gamma
    rss = a + b - np.sqrt(a * a + b * b)
    tot = (np.abs(g.r_u[:, 1:]) + np.abs(g.r_u[:, :-1]) + np.abs(g.r_v[1:]) + np.abs(g.r_v[:-1]) + np.abs(rss))
    return (tot > threshold).astype(float)


def fascd_vcycle(g: Level, thklim, finest=False, n_coarse=200, n_smooth=10, n_local_outer=10, n_local=10,
                 err_threshold=0.01):
    """FASCD V-cycle (glide/solver.py:71-157)."""
    if finest:
        g.w_u, g.w_v, g.w_H = g.u.copy(), g.v.copy(), g.H.copy()
        g.chi = g.gamma - g.H
    if g.child is None:
        g.gamma = g.w_H + g.chi
        g.vanka_sweep(n_coarse)
        g.gamma = np.full_like(g.gamma, thklim)
        return
    c = g.child
    c.chi = restrict_max_pool(g.chi)
    g.phi = prolong_cell_inject(-c.chi) + g.chi
    g.gamma = g.w_H + g.phi
    g.vanka_sweep(n_smooth)
    g.gamma = np.full_like(g.gamma, thklim)
    g.y_u, g.y_v, g.y_H = g.u - g.w_u, g.v - g.w_v, g.H - g.w_H
    c.u, c.v, c.H = restrict_u(g.u), restrict_v(g.v), restrict_cell(g.H)
    c.w_u, c.w_v, c.w_H = c.u.copy(), c.v.copy(), c.H.copy()
    g.compute_residual()
    cr_u, cr_v, cr_H = restrict_u(g.r_u), restrict_v(g.r_v), restrict_cell(g.r_H)
    F_u, F_v, F_H = c.compute_F()
    c.f_u, c.f_v, c.f_H = F_u - cr_u, F_v - cr_v, F_H - cr_H
    fascd_vcycle(c, thklim, n_coarse=n_coarse, n_smooth=n_smooth, n_local_outer=n_local_outer, n_local=n_local,
                 err_threshold=err_threshold)
    z_u = prolong_u_bilinear(c.u - c.w_u)
    z_v = prolong_v_bilinear(c.v - c.w_v)
    z_H = prolong_cell_inject(c.H - c.w_H)
    z_u, z_v, z_H = z_u + g.y_u, z_v + g.y_v, z_H + g.y_H
    g.u, g.v, g.H = g.w_u + z_u, g.w_v + z_v, g.w_H + z_H
    g.gamma = g.w_H + g.chi
    g.vanka_sweep(n_smooth)
    for _ in range(n_local_outer):
        g.error_mask = error_mask(g, err_threshold)
        g.vanka_sweep(n_local, local=True)
    g.gamma = np.full_like(g.gamma, thklim)


def adjoint_vcycle(g: Level, n_coarse=100, n_smooth=10):
    """Adjoint V-cycle (glide/solver.py:160-220)."""
    if g.child is None:
        g.compute_mask()
        g.vanka_sweep_adjoint(n_coarse, omega=1.0)
        g.mask = np.zeros_like(g.mask)
        return
    g.compute_mask()
    g.vanka_sweep_adjoint(n_smooth, omega=1.0)
    g.mask = np.zeros_like(g.mask)
    ra_u, ra_v, ra_H = g.adjoint_residual()
    c = g.child
    c.lu, c.lv, c.lH = restrict_u(g.lu), restrict_v(g.lv), restrict_cell(g.lH)
    restrict_parameters(g)
    c.fa_u, c.fa_v, c.fa_H = restrict_u(ra_u), restrict_v(ra_v), restrict_cell(ra_H)
    c.lu, c.lv, c.lH = np.zeros_like(c.lu), np.zeros_like(c.lv), np.zeros_like(c.lH)
    adjoint_vcycle(c, n_coarse=n_coarse, n_smooth=n_smooth)
    g.lu = g.lu + prolong_u_bilinear(c.lu)
    g.lv = g.lv + prolong_v_bilinear(c.lv)
    g.lH = g.lH + prolong_cell_bilinear(c.lH)
    g.compute_mask()
    g.vanka_sweep_adjoint(n_smooth, omega=1.0)
    g.mask = np.zeros_like(g.mask)


def residual_norm(g: Level):
    """|r| = sqrt(|r_u|^2 + |r_v|^2 + |FB(r_H, H-gamma)|^2) (glide/physics.py:176-198)."""
    rss = g.compute_residual(fischer_burmeister=True)
    return float(np.sqrt(np.sum(g.r_u ** 2) + np.sum(g.r_v ** 2) + np.sum(rss ** 2)))


class OracleIcePhysics:
    """IcePhysics restated on the CPU in FP64 (glide/physics.py:49-242)."""

    def __init__(self, ny, nx, dx, n_levels=5, n=3.0, eps_reg=1e-5, thklim=0.1, water_drag=1e-3,
                 calving_rate=1.0, gl_sigmoid_c=0.1, gl_derivatives=False):
        self.thklim = float(thklim)
        p = Params(n=n, eps_reg=eps_reg, water_drag=water_drag, calving_rate=calving_rate,
                   gl_sigmoid_c=gl_sigmoid_c, gl_derivatives=gl_derivatives)
        self.grid = Level(ny, nx, dx, 1.0, p)
        self.grids = [self.grid]
        for _ in range(n_levels - 1):
            self.grids.append(self.grids[-1].spawn_child())

    def set_geometry(self, bed, thickness):
        g = self.grid
        g.bed = np.asarray(bed, float).copy()
        g.H = np.asarray(thickness, float).copy()
        g.H_prev = g.H.copy()
        g.gamma = np.full_like(g.H, self.thklim)
        for par, ch in zip(self.grids[:-1], self.grids[1:]):
            ch.bed = restrict_cell(par.bed)
            ch.H = restrict_cell(par.H)
            ch.H_prev = restrict_cell(par.H_prev)
            ch.gamma = np.full_like(ch.H, self.thklim)

    def set_parameters(self, B=None, beta=None, smb=None):
        g = self.grid
        if B is not None:
            B = np.asarray(B, float)
            g.B = np.full_like(g.H, float(B)) if B.ndim == 0 else B.copy()
        if beta is not None:
            g.beta = np.asarray(beta, float).copy()
        if smb is not None:
            g.smb = np.asarray(smb, float).copy()
        restrict_parameters_to_hierarchy(g)

    def forward(self, dt, n_vcycles=3, update_geometry=True, tol=None, max_vcycles=50, history=None):
        for g in self.grids:
            g.dt = float(dt)
        g = self.grid
        g.f_H = g.H_prev / g.dt + g.smb
        r0 = residual_norm(g) if (tol is not None or history is not None) else None
        if history is not None:
            history.append(1.0)
        n = max_vcycles if tol is not None else n_vcycles
        for _ in range(n):
            fascd_vcycle(g, self.thklim, finest=True)
            if r0 is not None:
                rel = residual_norm(g) / r0 if r0 > 0 else 0.0
                if history is not None:
                    history.append(rel)
                if tol is not None and rel <= tol:
                    break
        if update_geometry:
            g.H_prev = g.H.copy()
        return g.u, g.v, g.H

    def adjoint(self, dL_du, dL_dv, dL_dH, n_vcycles=2, exact_boundary=False):
        g = self.grid
        g.fa_u, g.fa_v, g.fa_H = -np.asarray(dL_du, float), -np.asarray(dL_dv, float), -np.asarray(dL_dH, float)
        g.lu, g.lv, g.lH = np.zeros_like(g.u), np.zeros_like(g.v), np.zeros_like(g.H)
        for _ in range(n_vcycles):
            adjoint_vcycle(g)
        return g.compute_grad_beta(exact_boundary=exact_boundary)
