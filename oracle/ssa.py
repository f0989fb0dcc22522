"""FP64 NumPy restatement of GLIDE's SSA operators (test infrastructure only).

This module is the CPU oracle that the CUDA kernels of ``glide_b200`` are
checked against.  It is imported only by ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg; the product path never calls it.

Every function restates one reference kernel, vectorised over the grid, with
the same clamped-index boundary semantics and the same boundary zeroing rules.
Citations are ``glide/<file>:<line>`` inside the reference project.

Grid layout (MAC staggered, ``glide/grid.py:1-8``):
    u  on vertical faces   shape (ny, nx+1)
    v  on horizontal faces shape (ny+1, nx)
    H and parameters on cells shape (ny, nx)
Row index i grows "down"; v > 0 points to row i-1 (``glide/cuda/flux.cu``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

RHO_RATIO = 0.917  # rho_ice / rho_water, glide/cuda/stress.cu:250


@dataclass
class Params:
    """PhysicsParams (glide/cuda/common.cu:240-247, glide/kernels.py:10-49)."""
    n: float = 3.0
    eps_reg: float = 1e-5
    water_drag: float = 1e-3
    calving_rate: float = 1.0
    gl_sigmoid_c: float = 0.1
    gl_derivatives: bool = False


# ---------------------------------------------------------------------------
# clamped accessors (glide/cuda/common.cu:78-125)
# ---------------------------------------------------------------------------

def _ij(shape):
    ny, nx = shape
    return np.arange(ny)[:, None], np.arange(nx)[None, :]


def gc(a, I, J):
    """get_cell: clamp i to [0,ny-1], j to [0,nx-1] (common.cu:106-111)."""
    ny, nx = a.shape
    return a[np.clip(I, 0, ny - 1), np.clip(J, 0, nx - 1)]


def gu(u, I, J):
    """get_vfacet: clamp i to [0,ny-1], j to [0,nx] (common.cu:78-83)."""
    ny, nx1 = u.shape
    return u[np.clip(I, 0, ny - 1), np.clip(J, 0, nx1 - 1)]


def gv(v, I, J):
    """get_hfacet: clamp i to [0,ny], j to [0,nx-1] (common.cu:92-97)."""
    ny1, nx = v.shape
    return v[np.clip(I, 0, ny1 - 1), np.clip(J, 0, nx - 1)]


def sigmoid(z, c):
    """Clamped logistic, c*z in [-20,20] (common.cu:67-70)."""
    s = np.clip(c * z, -20.0, 20.0)
    return 1.0 / (1.0 + np.exp(-s))


def sigmoid_deriv(z, c):
    """common.cu:73-76."""
    s = sigmoid(z, c)
    return c * s * (1.0 - s)


# ---------------------------------------------------------------------------
# viscosity (glide/cuda/viscosity.cu:4-112)
# ---------------------------------------------------------------------------

def viscosity(u, v, B, p: Params, dx, du=None, dv=None):
    """Cell viscosity eta = 0.5 B eps_II^((1-n)/2n); returns (eta, d_eta).

    eps_II = ux^2 + vy^2 + ux*vy + 1/4 sum_corners eps_xy^2 + eps_reg with the
    corner shear masked at domain edges (viscosity.cu:61-112).  With a tangent
    (du, dv) the forward-mode derivative of the dual version
    (viscosity.cu:4-59) is returned as d_eta, else d_eta is None.
    """
    ny, nx = B.shape
    I, J = _ij((ny, nx))
    dxi = 1.0 / dx
    glen = (1.0 - p.n) / (2.0 * p.n)

    def comp(uu, vv):
        ul = gu(uu, I, J); ur = gu(uu, I, J + 1)
        vt = gv(vv, I, J); vb = gv(vv, I + 1, J)
        ux = (ur - ul) * dxi
        vy = (vt - vb) * dxi
        m_tl = ((I > 0) & (J > 0)).astype(float)
        m_tr = ((I > 0) & (J < nx - 1)).astype(float)
        m_bl = ((I < ny - 1) & (J > 0)).astype(float)
        m_br = ((I < ny - 1) & (J < nx - 1)).astype(float)
        e_tl = 0.5 * ((gu(uu, I - 1, J) - ul) * dxi + (vt - gv(vv, I, J - 1)) * dxi) * m_tl
        e_tr = 0.5 * ((gu(uu, I - 1, J + 1) - ur) * dxi + (gv(vv, I, J + 1) - vt) * dxi) * m_tr
        e_bl = 0.5 * ((ul - gu(uu, I + 1, J)) * dxi + (vb - gv(vv, I + 1, J - 1)) * dxi) * m_bl
        e_br = 0.5 * ((ur - gu(uu, I + 1, J + 1)) * dxi + (gv(vv, I + 1, J + 1) - vb) * dxi) * m_br
        return ux, vy, (e_tl, e_tr, e_bl, e_br)

    ux, vy, es = comp(u, v)
    exy2 = 0.25 * sum(e * e for e in es)
    eII = ux * ux + vy * vy + ux * vy + exy2 + p.eps_reg
    eta = 0.5 * B * eII ** glen
    if du is None:
        return eta, None
    dux, dvy, des = comp(du, dv)  # linear in the tangent
    d_exy2 = 0.25 * sum(2.0 * e * de for e, de in zip(es, des))
    d_eII = 2 * ux * dux + 2 * vy * dvy + (ux * dvy + vy * dux) + d_exy2
    d_eta = 0.5 * B * (glen * eII ** (glen - 1.0) * d_eII)
    return eta, d_eta


def _pad_edge(a, k=2):
    return np.pad(a, k, mode="edge")


class _CellShift:
    """Clamped neighbour views of a cell field: S(di,dj)[i,j] = a[clamp(i+di), clamp(j+dj)]."""

    def __init__(self, a, k=3):
        self.k = k
        self.p = _pad_edge(a, k)
        self.ny, self.nx = a.shape

    def __call__(self, di, dj, rows=None, cols=None):
        ny = self.ny if rows is None else rows
        nx = self.nx if cols is None else cols
        k = self.k
        return self.p[k + di:k + di + ny, k + dj:k + dj + nx]


# ---------------------------------------------------------------------------
# local stress / drag / flux terms (glide/cuda/stress.cu, glide/cuda/flux.cu)
# each returns (res, dict of partials) with the boundary zeroing rules
# ---------------------------------------------------------------------------

def sigma_xx(ul, ur, vt, vb, etaH, dxi, valid):
    """stress.cu:43-66; zero where the cell column is outside [0,nx)."""
    exx = 2.0 * (ur - ul) * dxi + (vt - vb) * dxi
    pre = 2.0 * etaH * dxi
    w = valid.astype(float)
    return (2.0 * etaH * exx * w,
            dict(ul=-2.0 * pre * w, ur=2.0 * pre * w, vt=pre * w, vb=-pre * w, etaH=2.0 * exx * w))


def sigma_yy(ul, ur, vt, vb, etaH, dxi, valid):
    """stress.cu:78-102; zero where the cell row is outside [0,ny)."""
    eyy = (ur - ul) * dxi + 2.0 * (vt - vb) * dxi
    pre = 2.0 * etaH * dxi
    w = valid.astype(float)
    return (2.0 * etaH * eyy * w,
            dict(ul=-pre * w, ur=pre * w, vt=2.0 * pre * w, vb=-2.0 * pre * w, etaH=2.0 * eyy * w))


def sigma_xy(ut, ub, vl, vr, etaH, dxi, valid):
    """stress.cu:159-183; zero on boundary vertices."""
    exy = 0.5 * ((ut - ub) * dxi + (vr - vl) * dxi)
    pre = etaH * dxi
    w = valid.astype(float)
    return (2.0 * etaH * exy * w,
            dict(ut=pre * w, ub=-pre * w, vl=-pre * w, vr=pre * w, etaH=2.0 * exy * w))


def tau_b(vel, H1, H2, bed1, bed2, beta1, beta2, p: Params):
    """Basal drag on a face between cells 1 and 2 (stress.cu:244-276, 330-361).

    Returns res, d_vel, d_H1, d_H2, d_beta1, d_beta2.
    """
    c = p.gl_sigmoid_c
    z1 = bed1 + RHO_RATIO * H1
    z2 = bed2 + RHO_RATIO * H2
    g1 = sigmoid(z1, c)
    g2 = sigmoid(z2, c)
    be1 = g1 * beta1 + (1.0 - g1) * p.water_drag
    be2 = g2 * beta2 + (1.0 - g2) * p.water_drag
    be = 0.5 * (be1 + be2)
    res = -be * vel
    d_vel = -be
    d_b1 = -0.5 * g1 * vel
    d_b2 = -0.5 * g2 * vel
    if p.gl_derivatives:
        d_H1 = -0.5 * (RHO_RATIO * sigmoid_deriv(z1, c)) * (beta1 - p.water_drag) * vel
        d_H2 = -0.5 * (RHO_RATIO * sigmoid_deriv(z2, c)) * (beta2 - p.water_drag) * vel
    else:
        d_H1 = np.zeros_like(res)
        d_H2 = np.zeros_like(res)
    return res, d_vel, d_H1, d_H2, d_b1, d_b2


def tau_d(Hm, Hp, bedm, bedp, dxi, valid):
    """Driving stress H_avg*(S_p - S_m)/dx on a face (stress.cu:406-436, 481-510).

    For x-faces m=left, p=right; for y-faces m=bottom, p=top.  Returns res,
    d_Hm, d_Hp, zero on boundary faces.
    """
    w = valid.astype(float)
    Havg = 0.5 * (Hm + Hp)
    base_m = np.maximum(bedm, -RHO_RATIO * Hm)
    base_p = np.maximum(bedp, -RHO_RATIO * Hp)
    db_m = np.where(bedm > -RHO_RATIO * Hm, 0.0, -RHO_RATIO)
    db_p = np.where(bedp > -RHO_RATIO * Hp, 0.0, -RHO_RATIO)
    Sm = base_m + Hm
    Sp = base_p + Hp
    res = Havg * (Sp - Sm) * dxi
    d_m = 0.5 * (Sp - Sm) * dxi - Havg * (1.0 + db_m) * dxi
    d_p = 0.5 * (Sp - Sm) * dxi + Havg * (1.0 + db_p) * dxi
    return res * w, d_m * w, d_p * w


def hflux(u, Hl, Hr, valid):
    """Upwind x-flux H_avg*u - 0.5|u|(Hr-Hl) (flux.cu:39-64). Returns res,d_u,d_Hl,d_Hr."""
    w = valid.astype(float)
    Havg = 0.5 * (Hl + Hr)
    um = np.abs(u)
    us = np.copysign(1.0, u)
    res = Havg * u - 0.5 * um * (Hr - Hl)
    return res * w, (Havg - 0.5 * us * (Hr - Hl)) * w, 0.5 * (u + um) * w, 0.5 * (u - um) * w


def vflux(v, Ht, Hb, valid):
    """Upwind y-flux H_avg*v - 0.5|v|(Ht-Hb) (flux.cu:110-135). Returns res,d_v,d_Ht,d_Hb."""
    w = valid.astype(float)
    Havg = 0.5 * (Ht + Hb)
    vm = np.abs(v)
    vs = np.copysign(1.0, v)
    res = Havg * v - 0.5 * vm * (Ht - Hb)
    return res * w, (Havg - 0.5 * vs * (Ht - Hb)) * w, 0.5 * (v - vm) * w, 0.5 * (v + vm) * w


def calving(H, bed, p: Params, c=None):
    """Calving sink -c_r (1-g) H (flux.cu:187-211). Returns res, d_H."""
    c = p.gl_sigmoid_c if c is None else c
    z = bed + RHO_RATIO * H
    g = sigmoid(z, c)
    res = -p.calving_rate * (1.0 - g) * H
    dH = -p.calving_rate * (1.0 - g)
    if p.gl_derivatives:
        dH = dH + p.calving_rate * H * (RHO_RATIO * sigmoid_deriv(z, c))
    return res, dH


# ---------------------------------------------------------------------------
# residual and JVP (glide/cuda/residuals.cu:6-579)
# ---------------------------------------------------------------------------

class _Fields:
    """Shifted views of all state/parameter fields used by the stencils."""

    def __init__(self, u, v, H, bed, B, beta, p, dx):
        self.ny, self.nx = H.shape
        self.u, self.v, self.H = u, v, H
        self.bed, self.B, self.beta = bed, B, beta
        self.p = p
        self.dx = dx
        self.dxi = 1.0 / dx


def _eta_vertex(eta_s, H_s, di, dj, rows, cols):
    """0.25*(eta*H) over the 4 cells around vertex (i+di, j+dj)."""
    return 0.25 * (eta_s(di - 1, dj - 1, rows, cols) * H_s(di - 1, dj - 1, rows, cols)
                   + eta_s(di - 1, dj, rows, cols) * H_s(di - 1, dj, rows, cols)
                   + eta_s(di, dj - 1, rows, cols) * H_s(di, dj - 1, rows, cols)
                   + eta_s(di, dj, rows, cols) * H_s(di, dj, rows, cols))


def _vertex_valid(I, J, ny, nx):
    return (I > 0) & (I < ny) & (J > 0) & (J < nx)


def momentum_u(u, v, H, bed, B, beta, p, dx, eta, du=None, dv=None, dH=None, deta=None):
    """u-face momentum residual (without -f_u) and optionally its JVP.

    residuals.cu:90-189 (residual) and :380-477 (JVP).
    """
    ny, nx = H.shape
    dxi = 1.0 / dx
    I, J = _ij((ny, nx + 1))
    rows, cols = ny, nx + 1
    Hs, es = _CellShift(H), _CellShift(eta)
    bs, bes = _CellShift(bed), _CellShift(beta)
    U = lambda a, di, dj: gu(a, I + di, J + dj)
    V = lambda a, di, dj: gv(a, I + di, J + dj)
    tan = du is not None
    if tan:
        dHs, des = _CellShift(dH), _CellShift(deta)
    out = np.zeros((rows, cols))
    dout = np.zeros((rows, cols)) if tan else None

    # sigma_xx at cell (i,j): + ; at cell (i,j-1): -
    for sgn, dj, in ((1.0, 0), (-1.0, -1)):
        etaH = es(0, dj, rows, cols) * Hs(0, dj, rows, cols)
        ul, ur = U(u, 0, dj), U(u, 0, dj + 1)
        vt, vb = V(v, 0, dj), V(v, 1, dj)
        valid = (J + dj >= 0) & (J + dj < nx)
        res, d = sigma_xx(ul, ur, vt, vb, etaH, dxi, valid)
        out += sgn * res * dxi
        if tan:
            detaH = des(0, dj, rows, cols) * Hs(0, dj, rows, cols) + es(0, dj, rows, cols) * dHs(0, dj, rows, cols)
            dres = (d["ul"] * U(du, 0, dj) + d["ur"] * U(du, 0, dj + 1) + d["vt"] * V(dv, 0, dj)
                    + d["vb"] * V(dv, 1, dj) + d["etaH"] * detaH)
            dout += sgn * dres * dxi
    # sigma_xy at vertex (i,j): + ; at vertex (i+1,j): -
    for sgn, di in ((1.0, 0), (-1.0, 1)):
        etaH = _eta_vertex(es, Hs, di, 0, rows, cols)
        ut, ub = U(u, di - 1, 0), U(u, di, 0)
        vl, vr = V(v, di, -1), V(v, di, 0)
        valid = _vertex_valid(I + di, J, ny, nx)
        res, d = sigma_xy(ut, ub, vl, vr, etaH, dxi, valid)
        out += sgn * res * dxi
        if tan:
            detaH = _eta_vertex(des, Hs, di, 0, rows, cols) + _eta_vertex(es, dHs, di, 0, rows, cols)
            dres = (d["ut"] * U(du, di - 1, 0) + d["ub"] * U(du, di, 0) + d["vl"] * V(dv, di, -1)
                    + d["vr"] * V(dv, di, 0) + d["etaH"] * detaH)
            dout += sgn * dres * dxi
    # basal drag between cells (i,j-1) and (i,j) (clamped)
    res, d_u, d_H1, d_H2, _, _ = tau_b(u, Hs(0, -1, rows, cols), Hs(0, 0, rows, cols),
                                       bs(0, -1, rows, cols), bs(0, 0, rows, cols),
                                       bes(0, -1, rows, cols), bes(0, 0, rows, cols), p)
    out += res
    if tan:
        dout += d_u * du + d_H1 * dHs(0, -1, rows, cols) + d_H2 * dHs(0, 0, rows, cols)
    # driving stress
    valid = (J > 0) & (J < nx)
    res, dm, dp = tau_d(Hs(0, -1, rows, cols), Hs(0, 0, rows, cols), bs(0, -1, rows, cols), bs(0, 0, rows, cols),
                        dxi, valid)
    out -= res
    if tan:
        dout -= dm * dHs(0, -1, rows, cols) + dp * dHs(0, 0, rows, cols)
    return out, dout


def momentum_v(u, v, H, bed, B, beta, p, dx, eta, du=None, dv=None, dH=None, deta=None):
    """v-face momentum residual (without -f_v) and optionally its JVP.

    residuals.cu:191-290 (residual) and :479-577 (JVP).
    """
    ny, nx = H.shape
    dxi = 1.0 / dx
    I, J = _ij((ny + 1, nx))
    rows, cols = ny + 1, nx
    Hs, es = _CellShift(H), _CellShift(eta)
    bs, bes = _CellShift(bed), _CellShift(beta)
    U = lambda a, di, dj: gu(a, I + di, J + dj)
    V = lambda a, di, dj: gv(a, I + di, J + dj)
    tan = du is not None
    if tan:
        dHs, des = _CellShift(dH), _CellShift(deta)
    out = np.zeros((rows, cols))
    dout = np.zeros((rows, cols)) if tan else None

    # sigma_yy at cell (i-1,j): + ; at cell (i,j): -
    for sgn, di in ((1.0, -1), (-1.0, 0)):
        etaH = es(di, 0, rows, cols) * Hs(di, 0, rows, cols)
        ul, ur = U(u, di, 0), U(u, di, 1)
        vt, vb = V(v, di, 0), V(v, di + 1, 0)
        valid = (I + di >= 0) & (I + di < ny)
        res, d = sigma_yy(ul, ur, vt, vb, etaH, dxi, valid)
        out += sgn * res * dxi
        if tan:
            detaH = des(di, 0, rows, cols) * Hs(di, 0, rows, cols) + es(di, 0, rows, cols) * dHs(di, 0, rows, cols)
            dres = (d["ul"] * U(du, di, 0) + d["ur"] * U(du, di, 1) + d["vt"] * V(dv, di, 0)
                    + d["vb"] * V(dv, di + 1, 0) + d["etaH"] * detaH)
            dout += sgn * dres * dxi
    # sigma_xy at vertex (i,j): - ; at vertex (i,j+1): +
    for sgn, dj in ((-1.0, 0), (1.0, 1)):
        etaH = _eta_vertex(es, Hs, 0, dj, rows, cols)
        ut, ub = U(u, -1, dj), U(u, 0, dj)
        vl, vr = V(v, 0, dj - 1), V(v, 0, dj)
        valid = _vertex_valid(I, J + dj, ny, nx)
        res, d = sigma_xy(ut, ub, vl, vr, etaH, dxi, valid)
        out += sgn * res * dxi
        if tan:
            detaH = _eta_vertex(des, Hs, 0, dj, rows, cols) + _eta_vertex(es, dHs, 0, dj, rows, cols)
            dres = (d["ut"] * U(du, -1, dj) + d["ub"] * U(du, 0, dj) + d["vl"] * V(dv, 0, dj - 1)
                    + d["vr"] * V(dv, 0, dj) + d["etaH"] * detaH)
            dout += sgn * dres * dxi
    res, d_v, d_H1, d_H2, _, _ = tau_b(v, Hs(-1, 0, rows, cols), Hs(0, 0, rows, cols),
                                       bs(-1, 0, rows, cols), bs(0, 0, rows, cols),
                                       bes(-1, 0, rows, cols), bes(0, 0, rows, cols), p)
    out += res
    if tan:
        dout += d_v * dv + d_H1 * dHs(-1, 0, rows, cols) + d_H2 * dHs(0, 0, rows, cols)
    # driving stress: m = bottom cell (i,j), p = top cell (i-1,j)
    valid = (I > 0) & (I < ny)
    res, dm, dp = tau_d(Hs(0, 0, rows, cols), Hs(-1, 0, rows, cols), bs(0, 0, rows, cols), bs(-1, 0, rows, cols),
                        dxi, valid)
    out -= res
    if tan:
        dout -= dm * dHs(0, 0, rows, cols) + dp * dHs(-1, 0, rows, cols)
    return out, dout


def mass(u, v, H, bed, p, dx, dt, du=None, dv=None, dH=None):
    """Mass residual H/dt - calving - div q without -f_H (residuals.cu:50-84, 343-373)."""
    ny, nx = H.shape
    dxi = 1.0 / dx
    I, J = _ij((ny, nx))
    Hs = _CellShift(H)
    tan = du is not None
    rH = H / dt
    cres, cdH = calving(H, bed, p)
    rH = rH - cres
    ul, ur = gu(u, I, J), gu(u, I, J + 1)
    vt, vb = gv(v, I, J), gv(v, I + 1, J)
    ql, ql_u, ql_l, ql_r = hflux(ul, Hs(0, -1), H, (J > 0) & (J < nx))
    qr, qr_u, qr_l, qr_r = hflux(ur, H, Hs(0, 1), (J + 1 > 0) & (J + 1 < nx))
    qt, qt_v, qt_t, qt_b = vflux(vt, Hs(-1, 0), H, (I > 0) & (I < ny))
    qb, qb_v, qb_t, qb_b = vflux(vb, H, Hs(1, 0), (I + 1 > 0) & (I + 1 < ny))
    rH = rH - ql * dxi + qr * dxi + qt * dxi - qb * dxi
    drH = None
    if tan:
        dHs = _CellShift(dH)
        dul, dur = gu(du, I, J), gu(du, I, J + 1)
        dvt, dvb = gv(dv, I, J), gv(dv, I + 1, J)
        drH = dH / dt - cdH * dH
        drH = drH - (ql_u * dul + ql_l * dHs(0, -1) + ql_r * dH) * dxi
        drH = drH + (qr_u * dur + qr_l * dH + qr_r * dHs(0, 1)) * dxi
        drH = drH + (qt_v * dvt + qt_t * dHs(-1, 0) + qt_b * dH) * dxi
        drH = drH - (qb_v * dvb + qb_t * dH + qb_b * dHs(1, 0)) * dxi
    return rH, drH


def residual(u, v, H, f_u, f_v, f_H, bed, B, beta, mask, gamma, p: Params, dx, dt):
    """r = F(U) - f with the active-set row (residuals.cu:6-292)."""
    eta, _ = viscosity(u, v, B, p, dx)
    ru, _ = momentum_u(u, v, H, bed, B, beta, p, dx, eta)
    rv, _ = momentum_v(u, v, H, bed, B, beta, p, dx, eta)
    rH, _ = mass(u, v, H, bed, p, dx, dt)
    rH = rH - f_H
    rH = (1.0 - mask) * rH + mask * (H - gamma)
    return ru - f_u, rv - f_v, rH


def jvp(u, v, H, du, dv, dH, bed, B, beta, mask, gamma, p: Params, dx, dt):
    """J(U) d (residuals.cu:299-579)."""
    eta, deta = viscosity(u, v, B, p, dx, du, dv)
    _, ju = momentum_u(u, v, H, bed, B, beta, p, dx, eta, du, dv, dH, deta)
    _, jv = momentum_v(u, v, H, bed, B, beta, p, dx, eta, du, dv, dH, deta)
    _, jH = mass(u, v, H, bed, p, dx, dt, du, dv, dH)
    jH = (1.0 - mask) * jH + mask * dH
    return ju, jv, jH


# ---------------------------------------------------------------------------
# VJP (glide/cuda/residuals.cu:586-1023)
# ---------------------------------------------------------------------------

class _Acc:
    """Scatter accumulator with a 2-wide margin; out-of-domain targets are
    dropped at the end like the bounds-checked flush (residuals.cu:985-1021)."""

    M = 2

    def __init__(self, rows, cols):
        self.a = np.zeros((rows + 2 * self.M, cols + 2 * self.M))
        self.rows, self.cols = rows, cols

    def add(self, di, dj, val):
        r, c = val.shape
        M = self.M
        self.a[M + di:M + di + r, M + dj:M + dj + c] += val

    def get(self, fold=False):
        """Interior values; with ``fold`` the margin is added onto the edge
        rows/columns, i.e. a contribution aimed at a clamped out-of-domain
        read goes to the cell that was actually read."""
        M = self.M
        a = self.a.copy()
        if fold:
            a[M, :] += a[:M, :].sum(axis=0)
            a[M + self.rows - 1, :] += a[M + self.rows:, :].sum(axis=0)
            a[:, M] += a[:, :M].sum(axis=1)
            a[:, M + self.cols - 1] += a[:, M + self.cols:].sum(axis=1)
        return a[M:M + self.rows, M:M + self.cols].copy()


def vjp(u, v, H, lu, lv, lH, bed, B, beta, mask, gamma, p: Params, dx, dt, exact_boundary=False):
    """Lambda^T J as the reference computes it (residuals.cu:586-1023).

    With ``exact_boundary`` the H contributions that the reference drops at
    clamped boundary reads (non-zero only for gl_derivatives=True) are kept,
    which makes this the exact transpose of ``jvp``.

    The velocity-velocity block reuses the forward tangent with lambda as
    the direction (residuals.cu:709,731,762,796,853,875,905,938), the other
    blocks are explicit transposes; contributions aimed outside the domain
    are dropped (residuals.cu:994,1007,1018).
    """
    ny, nx = H.shape
    dxi = 1.0 / dx
    eta, deta = viscosity(u, v, B, p, dx, lu, lv)
    accH = _Acc(ny, nx)
    accU = _Acc(ny, nx + 1)
    accV = _Acc(ny + 1, nx)

    # (A) cell rows (residuals.cu:644-686)
    I, J = _ij((ny, nx))
    Hs = _CellShift(H)
    lHm = lH * (1.0 - mask)
    _, cdH = calving(H, bed, p)
    accH.add(0, 0, lHm / dt - lHm * cdH)
    ul, ur = gu(u, I, J), gu(u, I, J + 1)
    vt, vb = gv(v, I, J), gv(v, I + 1, J)
    _, ql_u, ql_l, ql_r = hflux(ul, Hs(0, -1), H, (J > 0) & (J < nx))
    accH.add(0, 0, -lHm * ql_r * dxi); accH.add(0, -1, -lHm * ql_l * dxi); accU.add(0, 0, -lHm * ql_u * dxi)
    _, qr_u, qr_l, qr_r = hflux(ur, H, Hs(0, 1), (J + 1 > 0) & (J + 1 < nx))
    accH.add(0, 0, lHm * qr_l * dxi); accH.add(0, 1, lHm * qr_r * dxi); accU.add(0, 1, lHm * qr_u * dxi)
    _, qt_v, qt_t, qt_b = vflux(vt, Hs(-1, 0), H, (I > 0) & (I < ny))
    accH.add(0, 0, lHm * qt_b * dxi); accH.add(-1, 0, lHm * qt_t * dxi); accV.add(0, 0, lHm * qt_v * dxi)
    _, qb_v, qb_t, qb_b = vflux(vb, H, Hs(1, 0), (I + 1 > 0) & (I + 1 < ny))
    accH.add(0, 0, -lHm * qb_t * dxi); accH.add(1, 0, -lHm * qb_b * dxi); accV.add(1, 0, -lHm * qb_v * dxi)
    accH.add(0, 0, lH * mask)

    # (B) u-face rows (residuals.cu:691-834)
    I, J = _ij((ny, nx + 1))
    rows, cols = ny, nx + 1
    es, des = _CellShift(eta), _CellShift(deta)
    bs, bes = _CellShift(bed), _CellShift(beta)
    U = lambda a, di, dj: gu(a, I + di, J + dj)
    V = lambda a, di, dj: gv(a, I + di, J + dj)
    lam = gu(lu, I, J)
    for sgn, dj in ((1.0, 0), (-1.0, -1)):
        Hc = Hs(0, dj, rows, cols)
        etaH = es(0, dj, rows, cols) * Hc
        valid = (J + dj >= 0) & (J + dj < nx)
        _, d = sigma_xx(U(u, 0, dj), U(u, 0, dj + 1), V(v, 0, dj), V(v, 1, dj), etaH, dxi, valid)
        t = (d["ul"] * U(lu, 0, dj) + d["ur"] * U(lu, 0, dj + 1) + d["vt"] * V(lv, 0, dj)
             + d["vb"] * V(lv, 1, dj) + d["etaH"] * (Hc * des(0, dj, rows, cols)))
        accU.add(0, 0, sgn * t * dxi)
        accH.add(0, dj, sgn * lam * d["etaH"] * es(0, dj, rows, cols) * dxi)
    for sgn, di in ((1.0, 0), (-1.0, 1)):
        etaH = _eta_vertex(es, Hs, di, 0, rows, cols)
        valid = _vertex_valid(I + di, J, ny, nx)
        _, d = sigma_xy(U(u, di - 1, 0), U(u, di, 0), V(v, di, -1), V(v, di, 0), etaH, dxi, valid)
        detaH = _eta_vertex(des, Hs, di, 0, rows, cols)
        t = (d["ut"] * U(lu, di - 1, 0) + d["ub"] * U(lu, di, 0) + d["vl"] * V(lv, di, -1)
             + d["vr"] * V(lv, di, 0) + d["etaH"] * detaH)
        accU.add(0, 0, sgn * t * dxi)
        k = sgn * lam * d["etaH"] * 0.25 * dxi
        accH.add(di - 1, -1, k * es(di - 1, -1, rows, cols))
        accH.add(di - 1, 0, k * es(di - 1, 0, rows, cols))
        accH.add(di, -1, k * es(di, -1, rows, cols))
        accH.add(di, 0, k * es(di, 0, rows, cols))
    _, d_u, d_H1, d_H2, _, _ = tau_b(u, Hs(0, -1, rows, cols), Hs(0, 0, rows, cols),
                                     bs(0, -1, rows, cols), bs(0, 0, rows, cols),
                                     bes(0, -1, rows, cols), bes(0, 0, rows, cols), p)
    accU.add(0, 0, lam * d_u)
    accH.add(0, -1, lam * d_H1)
    accH.add(0, 0, lam * d_H2)
    _, dm, dpp = tau_d(Hs(0, -1, rows, cols), Hs(0, 0, rows, cols), bs(0, -1, rows, cols), bs(0, 0, rows, cols),
                       dxi, (J > 0) & (J < nx))
    accH.add(0, -1, -lam * dm)
    accH.add(0, 0, -lam * dpp)

    # (C) v-face rows (residuals.cu:836-975)
    I, J = _ij((ny + 1, nx))
    rows, cols = ny + 1, nx
    U = lambda a, di, dj: gu(a, I + di, J + dj)
    V = lambda a, di, dj: gv(a, I + di, J + dj)
    lam = gv(lv, I, J)
    for sgn, di in ((1.0, -1), (-1.0, 0)):
        Hc = Hs(di, 0, rows, cols)
        etaH = es(di, 0, rows, cols) * Hc
        valid = (I + di >= 0) & (I + di < ny)
        _, d = sigma_yy(U(u, di, 0), U(u, di, 1), V(v, di, 0), V(v, di + 1, 0), etaH, dxi, valid)
        t = (d["ul"] * U(lu, di, 0) + d["ur"] * U(lu, di, 1) + d["vt"] * V(lv, di, 0)
             + d["vb"] * V(lv, di + 1, 0) + d["etaH"] * (Hc * des(di, 0, rows, cols)))
        accV.add(0, 0, sgn * t * dxi)
        accH.add(di, 0, sgn * lam * d["etaH"] * es(di, 0, rows, cols) * dxi)
    for sgn, dj in ((-1.0, 0), (1.0, 1)):
        etaH = _eta_vertex(es, Hs, 0, dj, rows, cols)
        valid = _vertex_valid(I, J + dj, ny, nx)
        _, d = sigma_xy(U(u, -1, dj), U(u, 0, dj), V(v, 0, dj - 1), V(v, 0, dj), etaH, dxi, valid)
        detaH = _eta_vertex(des, Hs, 0, dj, rows, cols)
        t = (d["ut"] * U(lu, -1, dj) + d["ub"] * U(lu, 0, dj) + d["vl"] * V(lv, 0, dj - 1)
             + d["vr"] * V(lv, 0, dj) + d["etaH"] * detaH)
        accV.add(0, 0, sgn * t * dxi)
        k = sgn * lam * d["etaH"] * 0.25 * dxi
        accH.add(-1, dj - 1, k * es(-1, dj - 1, rows, cols))
        accH.add(-1, dj, k * es(-1, dj, rows, cols))
        accH.add(0, dj - 1, k * es(0, dj - 1, rows, cols))
        accH.add(0, dj, k * es(0, dj, rows, cols))
    _, d_v, d_H1, d_H2, _, _ = tau_b(v, Hs(-1, 0, rows, cols), Hs(0, 0, rows, cols),
                                     bs(-1, 0, rows, cols), bs(0, 0, rows, cols),
                                     bes(-1, 0, rows, cols), bes(0, 0, rows, cols), p)
    accV.add(0, 0, lam * d_v)
    accH.add(-1, 0, lam * d_H1)
    accH.add(0, 0, lam * d_H2)
    _, dm, dpp = tau_d(Hs(0, 0, rows, cols), Hs(-1, 0, rows, cols), bs(0, 0, rows, cols), bs(-1, 0, rows, cols),
                       dxi, (I > 0) & (I < ny))
    accH.add(0, 0, -lam * dm)
    accH.add(-1, 0, -lam * dpp)
    return accU.get(), accV.get(), accH.get(fold=exact_boundary)


# ---------------------------------------------------------------------------
# basal-friction gradient (glide/cuda/grad.cu:1-74)
# ---------------------------------------------------------------------------

def grad_beta(u, v, H, lu, lv, bed, beta, p: Params, exact_boundary=False):
    """grad_beta[c] = sum over faces lambda_face * d tau_b / d beta_c.

    The reference adds a u-face's left-cell term only when j > 0 and its
    right-cell term only when j < nx-1 (grad.cu:52-53), and likewise for v
    (grad.cu:70-71); ``exact_boundary=False`` keeps that rule.  With
    ``exact_boundary=True`` every term goes to the (clamped) cell it came
    from, which is the exact transpose used by finite-difference checks.
    """
    ny, nx = H.shape
    g = np.zeros((ny, nx))
    I, J = _ij((ny, nx + 1))
    Hs, bs, bes = _CellShift(H), _CellShift(bed), _CellShift(beta)
    rows, cols = ny, nx + 1
    _, _, _, _, db1, db2 = tau_b(u, Hs(0, -1, rows, cols), Hs(0, 0, rows, cols), bs(0, -1, rows, cols),
                                 bs(0, 0, rows, cols), bes(0, -1, rows, cols), bes(0, 0, rows, cols), p)
    c1 = lu * db1  # to cell (i, j-1)
    c2 = lu * db2  # to cell (i, j)
    if exact_boundary:
        np.add.at(g, (np.broadcast_to(I, c1.shape), np.clip(J - 1, 0, nx - 1)), c1)
        np.add.at(g, (np.broadcast_to(I, c2.shape), np.clip(J, 0, nx - 1)), c2)
    else:
        g[:, :nx - 1] += c1[:, 1:nx]          # j in [1, nx-1] -> cell j-1 (j>0); j=nx -> cell nx-1
        g[:, nx - 1] += c1[:, nx]
        g[:, :nx - 1] += c2[:, :nx - 1]       # j < nx-1 -> cell j
    I, J = _ij((ny + 1, nx))
    rows, cols = ny + 1, nx
    _, _, _, _, db1, db2 = tau_b(v, Hs(-1, 0, rows, cols), Hs(0, 0, rows, cols), bs(-1, 0, rows, cols),
                                 bs(0, 0, rows, cols), bes(-1, 0, rows, cols), bes(0, 0, rows, cols), p)
    c1 = lv * db1  # to cell (i-1, j)
    c2 = lv * db2  # to cell (i, j)
    if exact_boundary:
        np.add.at(g, (np.clip(I - 1, 0, ny - 1), np.broadcast_to(J, c1.shape)), c1)
        np.add.at(g, (np.clip(I, 0, ny - 1), np.broadcast_to(J, c2.shape)), c2)
    else:
        g[:ny - 1, :] += c1[1:ny, :]
        g[ny - 1, :] += c1[ny, :]
        g[:ny - 1, :] += c2[:ny - 1, :]
    return g
