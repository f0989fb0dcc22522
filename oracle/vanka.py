"""FP64 NumPy restatement of GLIDE's cell-patch Vanka smoothers (test infrastructure).

``vanka_deltas`` restates ``vanka_smooth`` / ``vanka_smooth_local``
(glide/cuda/vanka.cu:3-439, :844-1295) and ``vanka_adjoint_color`` restates
``vanka_smooth_adjoint`` (glide/cuda/vanka.cu:441-840), vectorised over all
cells.  Each cell holds a 5x5 local system in the unknown order
(u_l, u_r, v_t, v_b, H_c), row-major J[row*5+col] as in the reference.
"""
from __future__ import annotations

import numpy as np

from .ssa import (Params, _CellShift, _ij, calving, gc, gu, gv, hflux, sigma_xx, sigma_xy, sigma_yy, tau_b,
                  tau_d, vflux, viscosity)

REF_TILE = 14    # active cells per reference block (glide/grid.py:182-188: stride 14)
REF_HALO = 1     # halo ring of the 16x16 reference block


def lu5_solve(A, b):
    """Unpivoted Doolittle LU solve of 5x5 systems, vectorised over cells.

    A: (25, ...) row-major, b: (5, ...).  Restates lu_5x5_solve
    (glide/cuda/common.cu:132-175) step for step.
    """
    LU = [[A[i * 5 + j].copy() for j in range(5)] for i in range(5)]
    for k in range(5):
        inv = 1.0 / LU[k][k]
        for i in range(k + 1, 5):
            LU[i][k] = LU[i][k] * inv
            for j in range(k + 1, 5):
                LU[i][j] = LU[i][j] - LU[i][k] * LU[k][j]
    y = [None] * 5
    y[0] = b[0]
    y[1] = b[1] - LU[1][0] * y[0]
    y[2] = b[2] - LU[2][0] * y[0] - LU[2][1] * y[1]
    y[3] = b[3] - LU[3][0] * y[0] - LU[3][1] * y[1] - LU[3][2] * y[2]
    y[4] = b[4] - LU[4][0] * y[0] - LU[4][1] * y[1] - LU[4][2] * y[2] - LU[4][3] * y[3]
    x = [None] * 5
    x[4] = y[4] / LU[4][4]
    x[3] = (y[3] - LU[3][4] * x[4]) / LU[3][3]
    x[2] = (y[2] - LU[2][3] * x[3] - LU[2][4] * x[4]) / LU[2][2]
    x[1] = (y[1] - LU[1][2] * x[2] - LU[1][3] * x[3] - LU[1][4] * x[4]) / LU[1][1]
    x[0] = (y[0] - LU[0][1] * x[1] - LU[0][2] * x[2] - LU[0][3] * x[3] - LU[0][4] * x[4]) / LU[0][0]
    return x


def lu5_solve_pivot(A, b, tiny=1e-14):
    """Row-pivoted LU solve of 5x5 systems, vectorised over cells; restates
    lu_5x5_solve_pivot (glide/cuda/common.cu:180-233): the largest |entry| of
    the column is the pivot (first one on ties), a pivot below ``tiny`` skips
    its elimination step, a diagonal below ``tiny`` in back substitution gives
    x = 0."""
    LU = [[np.array(A[i * 5 + j], dtype=float, copy=True) for j in range(5)] for i in range(5)]
    y = [np.array(b[i], dtype=float, copy=True) for i in range(5)]
    for k in range(4):
        p = np.full(LU[k][k].shape, k)
        best = np.abs(LU[k][k])
        for i in range(k + 1, 5):
            a = np.abs(LU[i][k])
            take = a > best
            best = np.where(take, a, best)
            p = np.where(take, i, p)
        for i in range(k + 1, 5):
            sw = p == i
            for j in range(5):
                LU[k][j], LU[i][j] = np.where(sw, LU[i][j], LU[k][j]), np.where(sw, LU[k][j], LU[i][j])
            y[k], y[i] = np.where(sw, y[i], y[k]), np.where(sw, y[k], y[i])
        piv = LU[k][k]
        live = np.abs(piv) >= tiny
        safe = np.where(live, piv, 1.0)
        for i in range(k + 1, 5):
            f = np.where(live, LU[i][k] / safe, LU[i][k])
            LU[i][k] = f
            for j in range(k + 1, 5):
                LU[i][j] = np.where(live, LU[i][j] - f * LU[k][j], LU[i][j])
    for i in range(1, 5):
        for j in range(i):
            y[i] = y[i] - LU[i][j] * y[j]
    x = [None] * 5
    for i in range(4, -1, -1):
        v = y[i]
        for j in range(i + 1, 5):
            v = v - LU[i][j] * x[j]
        d = LU[i][i]
        x[i] = np.where(np.abs(d) > tiny, v / np.where(np.abs(d) > tiny, d, 1.0), 0.0)
    return x


class _Frozen:
    """Neighbour values that stay fixed during a cell's local Newton loop."""

    def __init__(self, u, v, H, bed, B, beta, p: Params, dx):
        ny, nx = H.shape
        self.ny, self.nx = ny, nx
        I, J = _ij((ny, nx))
        self.I, self.J = I, J
        eta, _ = viscosity(u, v, B, p, dx)
        es = _CellShift(eta)
        Hs = _CellShift(H)
        bs = _CellShift(bed)
        bes = _CellShift(beta)
        self.eta = {(di, dj): es(di, dj) for di in (-1, 0, 1) for dj in (-1, 0, 1)}
        self.H = {(di, dj): Hs(di, dj) for di in (-1, 0, 1) for dj in (-1, 0, 1)}
        self.bed = {(di, dj): bs(di, dj) for di, dj in ((0, 0), (0, -1), (0, 1), (-1, 0), (1, 0))}
        self.beta = {(di, dj): bes(di, dj) for di, dj in ((0, 0), (0, -1), (0, 1), (-1, 0), (1, 0))}
        self.U = lambda di, dj: gu(u, I + di, J + dj)
        self.V = lambda di, dj: gv(v, I + di, J + dj)


def _assemble(fz: _Frozen, ul, ur, vt, vb, Hc, p: Params, dx, dt, with_res, f=None, thklim=None):
    """Local 5x5 Jacobian (and residual) of a cell patch (vanka.cu:56-411).

    Returns (J list of 25 arrays, r list of 5 arrays or None, mass-row
    parts needed by the adjoint variant).
    """
    ny, nx = fz.ny, fz.nx
    I, J = fz.I, fz.J
    dxi = 1.0 / dx
    Jm = [np.zeros((ny, nx)) for _ in range(25)]
    r = [np.zeros((ny, nx)) for _ in range(5)] if with_res else None
    H = fz.H
    eta = fz.eta
    if with_res:
        f_u, f_v, f_H = f
        r[0] = r[0] - gu(f_u, I, J)
        r[1] = r[1] - gu(f_u, I, J + 1)
        r[2] = r[2] - gv(f_v, I, J)
        r[3] = r[3] - gv(f_v, I + 1, J)
        r[4] = r[4] - gc(f_H, I, J)

    # --- mass row (vanka.cu:67-115)
    Jm[24] = Jm[24] + 1.0 / dt
    if with_res:
        r[4] = r[4] + Hc / dt
    cres, cdH = calving(Hc, fz.bed[(0, 0)], p)
    Jm[24] = Jm[24] - cdH
    if with_res:
        r[4] = r[4] - cres
    q, q_u, q_l, q_r = hflux(ul, H[(0, -1)], Hc, (J > 0) & (J < nx))
    Jm[20] = Jm[20] - q_u * dxi; Jm[24] = Jm[24] - q_r * dxi
    if with_res:
        r[4] = r[4] - q * dxi
    q, q_u, q_l, q_r = hflux(ur, Hc, H[(0, 1)], (J + 1 > 0) & (J + 1 < nx))
    Jm[21] = Jm[21] + q_u * dxi; Jm[24] = Jm[24] + q_l * dxi
    if with_res:
        r[4] = r[4] + q * dxi
    q, q_v, q_t, q_b = vflux(vt, H[(-1, 0)], Hc, (I > 0) & (I < ny))
    Jm[22] = Jm[22] + q_v * dxi; Jm[24] = Jm[24] + q_b * dxi
    if with_res:
        r[4] = r[4] + q * dxi
    q, q_v, q_t, q_b = vflux(vb, Hc, H[(1, 0)], (I + 1 > 0) & (I + 1 < ny))
    Jm[23] = Jm[23] - q_v * dxi; Jm[24] = Jm[24] - q_t * dxi
    if with_res:
        r[4] = r[4] - q * dxi
        active = (Hc - dt * r[4]) <= thklim            # vanka.cu:104-113
        for k in range(20, 24):
            Jm[k] = np.where(active, 0.0, Jm[k])
        Jm[24] = np.where(active, 1.0, Jm[24])
        r[4] = np.where(active, Hc - thklim, r[4])

    # --- cell normal stresses (vanka.cu:117-152)
    etaH_c = eta[(0, 0)] * Hc
    d, res = None, None
    res, d = sigma_xx(ul, ur, vt, vb, etaH_c, dxi, (J >= 0) & (J < nx))
    dH = d["etaH"] * eta[(0, 0)] * dxi
    if with_res:
        r[0] = r[0] + res * dxi
    Jm[0] += d["ul"] * dxi; Jm[1] += d["ur"] * dxi; Jm[2] += d["vt"] * dxi; Jm[3] += d["vb"] * dxi; Jm[4] += dH
    if with_res:
        r[1] = r[1] - res * dxi
    Jm[5] -= d["ul"] * dxi; Jm[6] -= d["ur"] * dxi; Jm[7] -= d["vt"] * dxi; Jm[8] -= d["vb"] * dxi; Jm[9] -= dH
    res, d = sigma_yy(ul, ur, vt, vb, etaH_c, dxi, (I >= 0) & (I < ny))
    dH = d["etaH"] * eta[(0, 0)] * dxi
    if with_res:
        r[2] = r[2] - res * dxi
    Jm[10] -= d["ul"] * dxi; Jm[11] -= d["ur"] * dxi; Jm[12] -= d["vt"] * dxi; Jm[13] -= d["vb"] * dxi; Jm[14] -= dH
    if with_res:
        r[3] = r[3] + res * dxi
    Jm[15] += d["ul"] * dxi; Jm[16] += d["ur"] * dxi; Jm[17] += d["vt"] * dxi; Jm[18] += d["vb"] * dxi; Jm[19] += dH

    # --- neighbour normal stresses (vanka.cu:154-208)
    res, d = sigma_xx(fz.U(0, -1), ul, fz.V(0, -1), fz.V(1, -1), eta[(0, -1)] * H[(0, -1)], dxi,
                      (J - 1 >= 0) & (J - 1 < nx))
    if with_res:
        r[0] = r[0] - res * dxi
    Jm[0] -= d["ur"] * dxi
    res, d = sigma_xx(ur, fz.U(0, 2), fz.V(0, 1), fz.V(1, 1), eta[(0, 1)] * H[(0, 1)], dxi,
                      (J + 1 >= 0) & (J + 1 < nx))
    if with_res:
        r[1] = r[1] + res * dxi
    Jm[6] += d["ul"] * dxi
    res, d = sigma_yy(fz.U(-1, 0), fz.U(-1, 1), fz.V(-1, 0), vt, eta[(-1, 0)] * H[(-1, 0)], dxi,
                      (I - 1 >= 0) & (I - 1 < ny))
    if with_res:
        r[2] = r[2] + res * dxi
    Jm[12] += d["vb"] * dxi
    res, d = sigma_yy(fz.U(1, 0), fz.U(1, 1), vb, fz.V(2, 0), eta[(1, 0)] * H[(1, 0)], dxi,
                      (I + 1 >= 0) & (I + 1 < ny))
    if with_res:
        r[3] = r[3] - res * dxi
    Jm[18] -= d["vt"] * dxi

    def vert_valid(di, dj):
        return (I + di > 0) & (I + di < ny) & (J + dj > 0) & (J + dj < nx)

    # --- corner shear stresses (vanka.cu:211-311)
    # top-left vertex (i,j): cells tl=(-1,-1), tr=(-1,0), bl=(0,-1), br=c
    etaH = 0.25 * (eta[(-1, -1)] * H[(-1, -1)] + eta[(-1, 0)] * H[(-1, 0)] + eta[(0, -1)] * H[(0, -1)]
                   + eta[(0, 0)] * Hc)
    res, d = sigma_xy(fz.U(-1, 0), ul, fz.V(0, -1), vt, etaH, dxi, vert_valid(0, 0))
    dH = d["etaH"] * 0.25 * eta[(0, 0)] * dxi
    if with_res:
        r[0] = r[0] + res * dxi
        r[2] = r[2] - res * dxi
    Jm[0] += d["ub"] * dxi; Jm[4] += dH
    Jm[12] -= d["vr"] * dxi; Jm[14] -= dH
    # top-right vertex (i,j+1): cells tl=(-1,0), tr=(-1,1), bl=c, br=(0,1)
    etaH = 0.25 * (eta[(-1, 0)] * H[(-1, 0)] + eta[(-1, 1)] * H[(-1, 1)] + eta[(0, 0)] * Hc
                   + eta[(0, 1)] * H[(0, 1)])
    res, d = sigma_xy(fz.U(-1, 1), ur, vt, fz.V(0, 1), etaH, dxi, vert_valid(0, 1))
    dH = d["etaH"] * 0.25 * eta[(0, 0)] * dxi
    if with_res:
        r[1] = r[1] + res * dxi
        r[2] = r[2] + res * dxi
    Jm[6] += d["ub"] * dxi; Jm[9] += dH
    Jm[12] += d["vl"] * dxi; Jm[14] += dH
    # bottom-left vertex (i+1,j): cells tl=(0,-1), tr=c, bl=(1,-1), br=(1,0)
    etaH = 0.25 * (eta[(0, -1)] * H[(0, -1)] + eta[(0, 0)] * Hc + eta[(1, -1)] * H[(1, -1)]
                   + eta[(1, 0)] * H[(1, 0)])
    res, d = sigma_xy(ul, fz.U(1, 0), fz.V(1, -1), vb, etaH, dxi, vert_valid(1, 0))
    dH = d["etaH"] * 0.25 * eta[(0, 0)] * dxi
    if with_res:
        r[0] = r[0] - res * dxi
        r[3] = r[3] - res * dxi
    Jm[0] -= d["ut"] * dxi; Jm[4] -= dH
    Jm[18] -= d["vr"] * dxi; Jm[19] -= dH
    # bottom-right vertex (i+1,j+1): cells tl=c, tr=(0,1), bl=(1,0), br=(1,1)
    etaH = 0.25 * (eta[(0, 0)] * Hc + eta[(0, 1)] * H[(0, 1)] + eta[(1, 0)] * H[(1, 0)]
                   + eta[(1, 1)] * H[(1, 1)])
    res, d = sigma_xy(ur, fz.U(1, 1), vb, fz.V(1, 1), etaH, dxi, vert_valid(1, 1))
    dH = d["etaH"] * 0.25 * eta[(0, 0)] * dxi
    if with_res:
        r[1] = r[1] - res * dxi
        r[3] = r[3] + res * dxi
    Jm[6] -= d["ut"] * dxi; Jm[9] -= dH
    Jm[18] += d["vl"] * dxi; Jm[19] += dH

    # --- basal drag (vanka.cu:314-364)
    bed, beta = fz.bed, fz.beta
    res, d_u, d_H1, d_H2, _, _ = tau_b(ul, H[(0, -1)], Hc, bed[(0, -1)], bed[(0, 0)], beta[(0, -1)], beta[(0, 0)], p)
    if with_res:
        r[0] = r[0] + res
    Jm[0] += d_u; Jm[4] += d_H2
    res, d_u, d_H1, d_H2, _, _ = tau_b(ur, Hc, H[(0, 1)], bed[(0, 0)], bed[(0, 1)], beta[(0, 0)], beta[(0, 1)], p)
    if with_res:
        r[1] = r[1] + res
    Jm[6] += d_u; Jm[9] += d_H1
    res, d_v, d_H1, d_H2, _, _ = tau_b(vt, H[(-1, 0)], Hc, bed[(-1, 0)], bed[(0, 0)], beta[(-1, 0)], beta[(0, 0)], p)
    if with_res:
        r[2] = r[2] + res
    Jm[12] += d_v; Jm[14] += d_H2
    res, d_v, d_H1, d_H2, _, _ = tau_b(vb, Hc, H[(1, 0)], bed[(0, 0)], bed[(1, 0)], beta[(0, 0)], beta[(1, 0)], p)
    if with_res:
        r[3] = r[3] + res
    Jm[18] += d_v; Jm[19] += d_H1

    # --- driving stress (vanka.cu:366-404)
    res, dm, dpp = tau_d(H[(0, -1)], Hc, bed[(0, -1)], bed[(0, 0)], dxi, (J > 0) & (J < nx))
    if with_res:
        r[0] = r[0] - res
    Jm[4] -= dpp
    res, dm, dpp = tau_d(Hc, H[(0, 1)], bed[(0, 0)], bed[(0, 1)], dxi, (J + 1 > 0) & (J + 1 < nx))
    if with_res:
        r[1] = r[1] - res
    Jm[9] -= dm
    # y-faces: m = bottom cell, p = top cell
    res, dm, dpp = tau_d(Hc, H[(-1, 0)], bed[(0, 0)], bed[(-1, 0)], dxi, (I > 0) & (I < ny))
    if with_res:
        r[2] = r[2] - res
    Jm[14] -= dm
    res, dm, dpp = tau_d(H[(1, 0)], Hc, bed[(1, 0)], bed[(0, 0)], dxi, (I + 1 > 0) & (I + 1 < ny))
    if with_res:
        r[3] = r[3] - res
    Jm[19] -= dpp
    return Jm, r


def vanka_deltas(u, v, H, f_u, f_v, f_H, bed, B, beta, gamma, p: Params, dx, dt, n_newton=10, cell_on=None,
                 shift=1.0, return_cells=False, step=0.25, pivot=False):
    """Delta arrays written by one ``vanka_smooth`` launch (vanka.cu:3-439).

    Each cell runs ``n_newton`` damped (0.25) Newton steps on its 5 unknowns
    with neighbours and eta frozen, the momentum diagonals shifted by -1 and
    the mass diagonal by +1 (vanka.cu:406-410), H clamped to gamma
    (vanka.cu:423).  Faces receive 0.5*(change) from each adjacent cell
    (vanka.cu:433-436), H the full change.  ``cell_on`` (bool (ny,nx))
    restricts the update to those cells, as the block gating of
    ``vanka_smooth_local`` does.  ``step`` is the Newton step fraction
    (0.25 = relaxation_factor, vanka.cu:416; other values test the
    extension entry point glide_vanka_sweeps_ex); ``pivot`` solves the local
    systems with ``lu5_solve_pivot``.
    """
    ny, nx = H.shape
    fz = _Frozen(u, v, H, bed, B, beta, p, dx)
    ul0, ur0, vt0, vb0 = fz.U(0, 0), fz.U(0, 1), fz.V(0, 0), fz.V(1, 0)
    Hc0 = H.copy()
    ul, ur, vt, vb, Hc = ul0.copy(), ur0.copy(), vt0.copy(), vb0.copy(), Hc0.copy()
    thklim = gamma
    for _ in range(n_newton):
        Jm, r = _assemble(fz, ul, ur, vt, vb, Hc, p, dx, dt, True, (f_u, f_v, f_H), thklim)
        Jm[0] -= shift; Jm[6] -= shift; Jm[12] -= shift; Jm[18] -= shift; Jm[24] += shift
        x = lu5_solve_pivot(Jm, r) if pivot else lu5_solve(Jm, r)
        ul = ul - step * x[0]
        ur = ur - step * x[1]
        vt = vt - step * x[2]
        vb = vb - step * x[3]
        Hc = Hc - step * x[4]
        Hc = np.maximum(Hc, thklim)
    on = np.ones((ny, nx), bool) if cell_on is None else cell_on
    d_ul = np.where(on, 0.5 * (ul - ul0), 0.0)
    d_ur = np.where(on, 0.5 * (ur - ur0), 0.0)
    d_vt = np.where(on, 0.5 * (vt - vt0), 0.0)
    d_vb = np.where(on, 0.5 * (vb - vb0), 0.0)
    if return_cells:
        return d_ul, d_ur, d_vt, d_vb, np.where(on, Hc - Hc0, 0.0)
    du = np.zeros((ny, nx + 1)); dv = np.zeros((ny + 1, nx))
    du[:, :nx] += d_ul
    du[:, 1:] += d_ur
    dv[:ny, :] += d_vt
    dv[1:, :] += d_vb
    dH = np.where(on, Hc - Hc0, 0.0)
    return du, dv, dH


def vanka_linear_update(u, v, H, f_H, rho_u, rho_v, rho_H, d_H, bed, B, beta, gamma, p: Params, dx, dt,
                        shift=1.0):
    """One additive linear Vanka update for r + J d = 0 (test oracle of the
    extension entry point glide_vanka_linear, which has no counterpart in the
    reference).  Every cell solves its local matrix at (u, v, H) -- the matrix
    of the first local Newton iteration of vanka_deltas, with the same
    diagonal shift and with f_H in the mass row's active-set test -- against
    rho at its 4 faces and its cell; faces receive
    half of each adjacent cell's update, H the whole of it, bounded so that
    H + d_H + delta_H >= gamma.  Returns (du, dv, dH) before the omega factor.
    """
    ny, nx = H.shape
    fz = _Frozen(u, v, H, bed, B, beta, p, dx)
    zu, zv = np.zeros((ny, nx + 1)), np.zeros((ny + 1, nx))
    Jm, _ = _assemble(fz, fz.U(0, 0), fz.U(0, 1), fz.V(0, 0), fz.V(1, 0), H.copy(), p, dx, dt, True, (zu, zv, f_H),
                      gamma)
    Jm[0] -= shift; Jm[6] -= shift; Jm[12] -= shift; Jm[18] -= shift; Jm[24] += shift
    b = [rho_u[:, :nx], rho_u[:, 1:], rho_v[:ny], rho_v[1:], rho_H]
    x = lu5_solve(Jm, b)
    dH = np.maximum(-x[4], gamma - H - d_H)
    du = np.zeros((ny, nx + 1)); dv = np.zeros((ny + 1, nx))
    du[:, :nx] += -0.5 * x[0]
    du[:, 1:] += -0.5 * x[1]
    dv[:ny, :] += -0.5 * x[2]
    dv[1:, :] += -0.5 * x[3]
    return du, dv, dH


def local_cell_on(error_mask):
    """Cells updated by ``vanka_smooth_local`` (vanka.cu:875-888).

    A reference block updates its 14x14 active cells when any in-domain cell
    of its 16x16 window (active cells plus one ring) has error_mask > 0.5.
    """
    ny, nx = error_mask.shape
    bad = error_mask > 0.5
    on = np.zeros((ny, nx), bool)
    nby = ny // REF_TILE + 1
    nbx = nx // REF_TILE + 1
    for by in range(nby):
        i0 = by * REF_TILE
        if i0 >= ny:
            continue
        for bx in range(nbx):
            j0 = bx * REF_TILE
            if j0 >= nx:
                continue
            wi0, wi1 = max(i0 - REF_HALO, 0), min(i0 + REF_TILE + REF_HALO, ny)
            wj0, wj1 = max(j0 - REF_HALO, 0), min(j0 + REF_TILE + REF_HALO, nx)
            if bad[wi0:wi1, wj0:wj1].any():
                on[i0:min(i0 + REF_TILE, ny), j0:min(j0 + REF_TILE, nx)] = True
    return on


def vanka_adjoint_color(lu, lv, lH, mask, r_adj, u, v, H, bed, B, beta, gamma, p: Params, dx, dt, color,
                        omega=1.0):
    """One colour of ``vanka_smooth_adjoint`` (vanka.cu:441-840).

    Cells with (i+j)%2 == color solve J^T dlam = r_adj with the local
    Jacobian at the current state (rows of masked cells replaced by the
    identity, vanka.cu:534-538, no diagonal shift) and write
    lam_face + 0.5*omega*dlam, lam_H + omega*dlam (vanka.cu:834-838).
    Returns new (lu, lv, lH).
    """
    ny, nx = H.shape
    fz = _Frozen(u, v, H, bed, B, beta, p, dx)
    I, J = fz.I, fz.J
    ul, ur, vt, vb = fz.U(0, 0), fz.U(0, 1), fz.V(0, 0), fz.V(1, 0)
    Jm, _ = _assemble(fz, ul, ur, vt, vb, H, p, dx, dt, False)
    m = mask > 0.5
    for k in range(20, 24):
        Jm[k] = np.where(m, 0.0, Jm[k])
    Jm[24] = np.where(m, 1.0, Jm[24])
    JT = [Jm[c * 5 + rr] for rr in range(5) for c in range(5)]
    ru, rv, rH = r_adj
    rhs = [gu(ru, I, J), gu(ru, I, J + 1), gv(rv, I, J), gv(rv, I + 1, J), rH]
    x = lu5_solve(JT, rhs)
    sel = ((I + J) % 2) == color
    lu_o, lv_o, lH_o = lu.copy(), lv.copy(), lH.copy()
    # each face is adjacent to exactly one cell of each colour
    upd_l = lu[:, :nx] + 0.5 * omega * x[0]
    upd_r = lu[:, 1:] + 0.5 * omega * x[1]
    lu_o[:, :nx] = np.where(sel, upd_l, lu_o[:, :nx])
    lu_o[:, 1:] = np.where(sel, upd_r, lu_o[:, 1:])
    upd_t = lv[:ny, :] + 0.5 * omega * x[2]
    upd_b = lv[1:, :] + 0.5 * omega * x[3]
    lv_o[:ny, :] = np.where(sel, upd_t, lv_o[:ny, :])
    lv_o[1:, :] = np.where(sel, upd_b, lv_o[1:, :])
    lH_o = np.where(sel, lH + omega * x[4], lH_o)
    return lu_o, lv_o, lH_o
