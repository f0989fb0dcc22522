// Cell-patch Vanka smoothers (glide/cuda/vanka.cu) on B200.
//
// Forward sweep = two kernels:
//   vanka_cells: one thread per cell runs the damped local Newton iterations
//     on the cell's 5 unknowns (u_l, u_r, v_t, v_b, H_c) with the neighbours
//     and the viscosity frozen, and stores half of each face change and the
//     full H change per cell (deterministic, no atomics);
//   vanka_apply: every face adds the halves of its two cells, U += omega*delta
//     (the reference zero-fills a delta vector, scatters with atomicAdd and
//     axpys on the host: glide/grid.py:305-317, vanka.cu:433-437).
// The viscosity of the tile plus a one-cell ring is computed once into shared
// memory; the neighbours' grounding sigmoids are hoisted out of the Newton
// loop.  The local variant gates cells by the reference's 16x16-window /
// stride-14 block rule (vanka.cu:875-888) through per-tile flags.
#include "glide_common.cuh"

namespace glide {

constexpr int VX = 32, VY = 8, VNT = VX * VY;
constexpr int REF_STRIDE = 14;   // reference block stride (glide/grid.py:182-188)
constexpr int REF_WIN = 16;      // reference block (active cells + 1 ring)

// Everything a cell patch needs from outside its 5 unknowns.
template <typename T> struct Patch {
    T eta[3][3];                 // eta at (i-1..i+1, j-1..j+1)
    T Hn[3][3];                  // H at the same cells ([1][1] unused: iterated)
    T bed_c, bed_l, bed_r, bed_t, bed_b;
    T beta_c, beta_l, beta_r, beta_t, beta_b;
    T g_l, g_r, g_t, g_b;        // grounded fractions of the 4 neighbours (frozen)
    T u_ll, u_rr, u_tl, u_tr, u_bl, u_br;
    T v_lt, v_lb, v_rt, v_rb, v_tt, v_bb;
    int i, j;
};

// Local 5x5 Jacobian and residual of cell (i,j) at the local iterate
// (vanka.cu:56-404).  Row/column order (u_l, u_r, v_t, v_b, H_c).
// WITH_RES adds the residual and the active-set switch (vanka.cu:104-113);
// the adjoint variant calls it without.
template <typename T, bool WITH_RES>
__device__ __forceinline__ void assemble(const Patch<T>& P, T ul, T ur, T vt, T vb, T Hc, T fu_l, T fu_r, T fv_t,
                                         T fv_b, T fH, T thklim, int ny, int nx, const Phys<T>& p, T (&J)[25],
                                         T (&r)[5]) {
    const int i = P.i, j = P.j;
    const T dxi = p.dxi;
#pragma unroll
    for (int k = 0; k < 25; k++) J[k] = T(0);
    if (WITH_RES) {
        r[0] = -fu_l; r[1] = -fu_r; r[2] = -fv_t; r[3] = -fv_b; r[4] = -fH;
    }
    const T gc = sigmoid(P.bed_c + rho_ratio<T>() * Hc, p.sig_c);

    // mass row (vanka.cu:67-115)
    {
        J[24] = T(1) / p.dt;
        if (WITH_RES) r[4] += Hc / p.dt;
        Calving<T> cv = calving_g(Hc, gc, p);
        J[24] -= cv.d_H;
        if (WITH_RES) r[4] -= cv.res;
        Flux<T> ql = upwind_flux(ul, P.Hn[1][0], Hc, j > 0 && j < nx);
        J[20] -= ql.d_vel * dxi; J[24] -= ql.d_Hb * dxi;
        if (WITH_RES) r[4] -= ql.res * dxi;
        Flux<T> qr = upwind_flux(ur, Hc, P.Hn[1][2], j + 1 > 0 && j + 1 < nx);
        J[21] += qr.d_vel * dxi; J[24] += qr.d_Ha * dxi;
        if (WITH_RES) r[4] += qr.res * dxi;
        Flux<T> qt = upwind_flux(vt, Hc, P.Hn[0][1], i > 0 && i < ny);
        J[22] += qt.d_vel * dxi; J[24] += qt.d_Ha * dxi;
        if (WITH_RES) r[4] += qt.res * dxi;
        Flux<T> qb = upwind_flux(vb, P.Hn[2][1], Hc, i + 1 > 0 && i + 1 < ny);
        J[23] -= qb.d_vel * dxi; J[24] -= qb.d_Hb * dxi;
        if (WITH_RES) {
            r[4] -= qb.res * dxi;
            if ((Hc - p.dt * r[4]) <= thklim) {
                J[20] = T(0); J[21] = T(0); J[22] = T(0); J[23] = T(0);
                J[24] = T(1);
                r[4] = Hc - thklim;
            }
        }
    }
    const T (&eta)[3][3] = P.eta;
    // own-cell normal stresses (vanka.cu:117-152)
    {
        const T etaH = eta[1][1] * Hc;
        NormalStress<T> s = normal_stress<T, true>(ul, ur, vt, vb, etaH, dxi, true);
        const T dH = s.d_etaH * eta[1][1] * dxi;
        if (WITH_RES) { r[0] += s.res * dxi; r[1] -= s.res * dxi; }
        J[0] += s.d_ul * dxi; J[1] += s.d_ur * dxi; J[2] += s.d_vt * dxi; J[3] += s.d_vb * dxi; J[4] += dH;
        J[5] -= s.d_ul * dxi; J[6] -= s.d_ur * dxi; J[7] -= s.d_vt * dxi; J[8] -= s.d_vb * dxi; J[9] -= dH;
        NormalStress<T> y = normal_stress<T, false>(ul, ur, vt, vb, etaH, dxi, true);
        const T dHy = y.d_etaH * eta[1][1] * dxi;
        if (WITH_RES) { r[2] -= y.res * dxi; r[3] += y.res * dxi; }
        J[10] -= y.d_ul * dxi; J[11] -= y.d_ur * dxi; J[12] -= y.d_vt * dxi; J[13] -= y.d_vb * dxi; J[14] -= dHy;
        J[15] += y.d_ul * dxi; J[16] += y.d_ur * dxi; J[17] += y.d_vt * dxi; J[18] += y.d_vb * dxi; J[19] += dHy;
    }
    // neighbour normal stresses (vanka.cu:154-208)
    {
        NormalStress<T> s = normal_stress<T, true>(P.u_ll, ul, P.v_lt, P.v_lb, eta[1][0] * P.Hn[1][0], dxi, j - 1 >= 0);
        if (WITH_RES) r[0] -= s.res * dxi;
        J[0] -= s.d_ur * dxi;
        s = normal_stress<T, true>(ur, P.u_rr, P.v_rt, P.v_rb, eta[1][2] * P.Hn[1][2], dxi, j + 1 < nx);
        if (WITH_RES) r[1] += s.res * dxi;
        J[6] += s.d_ul * dxi;
        s = normal_stress<T, false>(P.u_tl, P.u_tr, P.v_tt, vt, eta[0][1] * P.Hn[0][1], dxi, i - 1 >= 0);
        if (WITH_RES) r[2] += s.res * dxi;
        J[12] += s.d_vb * dxi;
        s = normal_stress<T, false>(P.u_bl, P.u_br, vb, P.v_bb, eta[2][1] * P.Hn[2][1], dxi, i + 1 < ny);
        if (WITH_RES) r[3] -= s.res * dxi;
        J[18] -= s.d_vt * dxi;
    }
    // corner shear stresses (vanka.cu:211-311)
    {
        const T ec = T(0.25) * eta[1][1];
        // top-left vertex (i,j)
        T etaH = T(0.25) * (eta[0][0] * P.Hn[0][0] + eta[0][1] * P.Hn[0][1] + eta[1][0] * P.Hn[1][0]) + ec * Hc;
        ShearStress<T> s = shear_stress(P.u_tl, ul, P.v_lt, vt, etaH, dxi, i > 0 && j > 0);
        if (WITH_RES) { r[0] += s.res * dxi; r[2] -= s.res * dxi; }
        J[0] += s.d_ub * dxi; J[4] += s.d_etaH * ec * dxi;
        J[12] -= s.d_vr * dxi; J[14] -= s.d_etaH * ec * dxi;
        // top-right vertex (i,j+1)
        etaH = T(0.25) * (eta[0][1] * P.Hn[0][1] + eta[0][2] * P.Hn[0][2] + eta[1][2] * P.Hn[1][2]) + ec * Hc;
        s = shear_stress(P.u_tr, ur, vt, P.v_rt, etaH, dxi, i > 0 && j + 1 < nx);
        if (WITH_RES) { r[1] += s.res * dxi; r[2] += s.res * dxi; }
        J[6] += s.d_ub * dxi; J[9] += s.d_etaH * ec * dxi;
        J[12] += s.d_vl * dxi; J[14] += s.d_etaH * ec * dxi;
        // bottom-left vertex (i+1,j)
        etaH = T(0.25) * (eta[1][0] * P.Hn[1][0] + eta[2][0] * P.Hn[2][0] + eta[2][1] * P.Hn[2][1]) + ec * Hc;
        s = shear_stress(ul, P.u_bl, P.v_lb, vb, etaH, dxi, i + 1 < ny && j > 0);
        if (WITH_RES) { r[0] -= s.res * dxi; r[3] -= s.res * dxi; }
        J[0] -= s.d_ut * dxi; J[4] -= s.d_etaH * ec * dxi;
        J[18] -= s.d_vr * dxi; J[19] -= s.d_etaH * ec * dxi;
        // bottom-right vertex (i+1,j+1)
        etaH = T(0.25) * (eta[1][2] * P.Hn[1][2] + eta[2][1] * P.Hn[2][1] + eta[2][2] * P.Hn[2][2]) + ec * Hc;
        s = shear_stress(ur, P.u_br, vb, P.v_rb, etaH, dxi, i + 1 < ny && j + 1 < nx);
        if (WITH_RES) { r[1] -= s.res * dxi; r[3] += s.res * dxi; }
        J[6] -= s.d_ut * dxi; J[9] -= s.d_etaH * ec * dxi;
        J[18] += s.d_vl * dxi; J[19] += s.d_etaH * ec * dxi;
    }
    // basal drag (vanka.cu:314-364)
    {
        BasalDrag<T> d = basal_drag_g(ul, P.g_l, gc, P.beta_l, P.beta_c, p);
        if (WITH_RES) r[0] += d.res;
        J[0] += d.d_vel; J[4] += d.d_H2;
        d = basal_drag_g(ur, gc, P.g_r, P.beta_c, P.beta_r, p);
        if (WITH_RES) r[1] += d.res;
        J[6] += d.d_vel; J[9] += d.d_H1;
        d = basal_drag_g(vt, P.g_t, gc, P.beta_t, P.beta_c, p);
        if (WITH_RES) r[2] += d.res;
        J[12] += d.d_vel; J[14] += d.d_H2;
        d = basal_drag_g(vb, gc, P.g_b, P.beta_c, P.beta_b, p);
        if (WITH_RES) r[3] += d.res;
        J[18] += d.d_vel; J[19] += d.d_H1;
    }
    // driving stress (vanka.cu:366-404); y-faces: m = bottom, p = top
    {
        Driving<T> d = driving(P.Hn[1][0], Hc, P.bed_l, P.bed_c, dxi, j > 0 && j < nx);
        if (WITH_RES) r[0] -= d.res;
        J[4] -= d.d_Hp;
        d = driving(Hc, P.Hn[1][2], P.bed_c, P.bed_r, dxi, j + 1 < nx);
        if (WITH_RES) r[1] -= d.res;
        J[9] -= d.d_Hm;
        d = driving(Hc, P.Hn[0][1], P.bed_c, P.bed_t, dxi, i > 0 && i < ny);
        if (WITH_RES) r[2] -= d.res;
        J[14] -= d.d_Hm;
        d = driving(P.Hn[2][1], Hc, P.bed_b, P.bed_c, dxi, i + 1 < ny);
        if (WITH_RES) r[3] -= d.res;
        J[19] -= d.d_Hp;
    }
}

// Fill the eta window of a VYxVX tile (+ ring) and the frozen patch of the
// calling thread's cell.
template <typename T>
__device__ __forceinline__ void eta_window(T (*s_eta)[VX + 2], const T* u, const T* v, const T* B, int i0, int j0,
                                           int ny, int nx, const Phys<T>& p) {
    for (int k = threadIdx.x; k < (VY + 2) * (VX + 2); k += VNT) {
        int r = k / (VX + 2), c = k - r * (VX + 2);
        int ic = clampi(i0 - 1 + r, 0, ny - 1), jc = clampi(j0 - 1 + c, 0, nx - 1);
        EtaIn<T> e = eta_inputs(u, v, ic, jc, ny, nx);
        s_eta[r][c] = cell_eta(e, ldc(B, ic, jc, ny, nx), ic, jc, ny, nx, p).eta;
    }
}

template <typename T>
__device__ __forceinline__ void load_patch(Patch<T>& P, T (*s_eta)[VX + 2], int r, int c, const T* u, const T* v,
                                           const T* H, const T* bed, const T* beta, int i, int j, int ny, int nx,
                                           const Phys<T>& p) {
    P.i = i;
    P.j = j;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            P.eta[a][b] = s_eta[r + a][c + b];
            P.Hn[a][b] = ldc(H, i - 1 + a, j - 1 + b, ny, nx);
        }
    P.bed_c = ldc(bed, i, j, ny, nx); P.bed_l = ldc(bed, i, j - 1, ny, nx); P.bed_r = ldc(bed, i, j + 1, ny, nx);
    P.bed_t = ldc(bed, i - 1, j, ny, nx); P.bed_b = ldc(bed, i + 1, j, ny, nx);
    P.beta_c = ldc(beta, i, j, ny, nx); P.beta_l = ldc(beta, i, j - 1, ny, nx); P.beta_r = ldc(beta, i, j + 1, ny, nx);
    P.beta_t = ldc(beta, i - 1, j, ny, nx); P.beta_b = ldc(beta, i + 1, j, ny, nx);
    P.g_l = sigmoid(P.bed_l + rho_ratio<T>() * P.Hn[1][0], p.sig_c);
    P.g_r = sigmoid(P.bed_r + rho_ratio<T>() * P.Hn[1][2], p.sig_c);
    P.g_t = sigmoid(P.bed_t + rho_ratio<T>() * P.Hn[0][1], p.sig_c);
    P.g_b = sigmoid(P.bed_b + rho_ratio<T>() * P.Hn[2][1], p.sig_c);
    P.u_ll = ldu(u, i, j - 1, ny, nx); P.u_rr = ldu(u, i, j + 2, ny, nx);
    P.u_tl = ldu(u, i - 1, j, ny, nx); P.u_tr = ldu(u, i - 1, j + 1, ny, nx);
    P.u_bl = ldu(u, i + 1, j, ny, nx); P.u_br = ldu(u, i + 1, j + 1, ny, nx);
    P.v_lt = ldv(v, i, j - 1, ny, nx); P.v_lb = ldv(v, i + 1, j - 1, ny, nx);
    P.v_rt = ldv(v, i, j + 1, ny, nx); P.v_rb = ldv(v, i + 1, j + 1, ny, nx);
    P.v_tt = ldv(v, i - 1, j, ny, nx); P.v_bb = ldv(v, i + 2, j, ny, nx);
}

__device__ __forceinline__ bool ref_tile_on(const int* flags, int i, int j, int nx) {
    const int nbx = nx / REF_STRIDE + 1;
    return flags[(i / REF_STRIDE) * nbx + j / REF_STRIDE] != 0;
}

// Frozen per-cell coefficients of the forward local Newton loop: every term
// that depends only on neighbour values (fixed during a cell's iterations) is
// evaluated once here, so the loop only evaluates what depends on the cell's
// own 5 unknowns.  Same formulas as assemble<T,true>; the neighbour normal
// stresses are kept as k*(x - x_far) + c so no cancellation is introduced.
template <typename T> struct Frozen {
    T eta_c, ec;                       // eta of the cell, 0.25*eta
    T kl, cl, u_ll, kr, cr, u_rr;      // sxx of left/right cell
    T kt, ct, v_tt, kb, cb, v_bb;      // syy of top/bottom cell
    T S_tl, S_tr, S_bl, S_br;          // 0.25 * sum of the 3 frozen eta*H around each vertex
    T u_tl, v_lt, u_tr, v_rt, u_bl, v_lb, u_br, v_rb;
    T w_tl, w_tr, w_bl, w_br;          // vertex validity (0/1)
    T be_l, be_r, be_t, be_b;          // neighbour half of beta_eff: g*beta + (1-g)*wd
    T g_l, g_r, g_t, g_b;              // neighbour grounded fractions (gl_derivatives only)
    T beta_l, beta_r, beta_t, beta_b;
    T H_l, H_r, H_t, H_b;
    T S_l, S_r, S_t, S_b;              // neighbour surfaces max(bed,-0.917H)+H
    T db_l, db_r, db_t, db_b;          // 1 + dbase/dH of the neighbours
    T w_l, w_r, w_t, w_b;              // flux / driving validity of the 4 faces
    T bed_c, beta_c;
};

template <typename T>
__device__ __forceinline__ void make_frozen(Frozen<T>& F, const Patch<T>& P, int ny, int nx, const Phys<T>& p) {
    const int i = P.i, j = P.j;
    const T dxi = p.dxi;
    const T (&eta)[3][3] = P.eta;
    const T (&Hn)[3][3] = P.Hn;
    F.eta_c = eta[1][1];
    F.ec = T(0.25) * eta[1][1];
    T wl = (j - 1 >= 0) ? T(1) : T(0), wr = (j + 1 < nx) ? T(1) : T(0);
    T wt = (i - 1 >= 0) ? T(1) : T(0), wb = (i + 1 < ny) ? T(1) : T(0);
    T eHl = eta[1][0] * Hn[1][0], eHr = eta[1][2] * Hn[1][2], eHt = eta[0][1] * Hn[0][1], eHb = eta[2][1] * Hn[2][1];
    F.kl = T(4) * eHl * dxi * wl;  F.cl = T(2) * eHl * dxi * wl * (P.v_lt - P.v_lb);  F.u_ll = P.u_ll;
    F.kr = T(4) * eHr * dxi * wr;  F.cr = T(2) * eHr * dxi * wr * (P.v_rt - P.v_rb);  F.u_rr = P.u_rr;
    F.kt = T(4) * eHt * dxi * wt;  F.ct = T(2) * eHt * dxi * wt * (P.u_tr - P.u_tl);  F.v_tt = P.v_tt;
    F.kb = T(4) * eHb * dxi * wb;  F.cb = T(2) * eHb * dxi * wb * (P.u_br - P.u_bl);  F.v_bb = P.v_bb;
    F.S_tl = T(0.25) * (eta[0][0] * Hn[0][0] + eHt + eHl);
    F.S_tr = T(0.25) * (eHt + eta[0][2] * Hn[0][2] + eHr);
    F.S_bl = T(0.25) * (eHl + eta[2][0] * Hn[2][0] + eHb);
    F.S_br = T(0.25) * (eHr + eHb + eta[2][2] * Hn[2][2]);
    F.u_tl = P.u_tl; F.v_lt = P.v_lt; F.u_tr = P.u_tr; F.v_rt = P.v_rt;
    F.u_bl = P.u_bl; F.v_lb = P.v_lb; F.u_br = P.u_br; F.v_rb = P.v_rb;
    F.w_tl = (i > 0 && j > 0) ? T(1) : T(0);
    F.w_tr = (i > 0 && j + 1 < nx) ? T(1) : T(0);
    F.w_bl = (i + 1 < ny && j > 0) ? T(1) : T(0);
    F.w_br = (i + 1 < ny && j + 1 < nx) ? T(1) : T(0);
    F.g_l = P.g_l; F.g_r = P.g_r; F.g_t = P.g_t; F.g_b = P.g_b;
    F.beta_l = P.beta_l; F.beta_r = P.beta_r; F.beta_t = P.beta_t; F.beta_b = P.beta_b;
    F.be_l = P.g_l * P.beta_l + (T(1) - P.g_l) * p.water_drag;
    F.be_r = P.g_r * P.beta_r + (T(1) - P.g_r) * p.water_drag;
    F.be_t = P.g_t * P.beta_t + (T(1) - P.g_t) * p.water_drag;
    F.be_b = P.g_b * P.beta_b + (T(1) - P.g_b) * p.water_drag;
    F.H_l = Hn[1][0]; F.H_r = Hn[1][2]; F.H_t = Hn[0][1]; F.H_b = Hn[2][1];
    auto surf = [&](T bed, T H, T& S, T& db) {
        S = M<T>::max(bed, -rho_ratio<T>() * H) + H;
        db = T(1) + (bed > -rho_ratio<T>() * H ? T(0) : -rho_ratio<T>());
    };
    surf(P.bed_l, F.H_l, F.S_l, F.db_l);
    surf(P.bed_r, F.H_r, F.S_r, F.db_r);
    surf(P.bed_t, F.H_t, F.S_t, F.db_t);
    surf(P.bed_b, F.H_b, F.S_b, F.db_b);
    F.w_l = (j > 0 && j < nx) ? T(1) : T(0);
    F.w_r = (j + 1 < nx) ? T(1) : T(0);
    F.w_t = (i > 0 && i < ny) ? T(1) : T(0);
    F.w_b = (i + 1 < ny) ? T(1) : T(0);
    F.bed_c = P.bed_c;
    F.beta_c = P.beta_c;
}

// One local Newton step's matrix and residual from the frozen coefficients
// (same terms and order of rows/columns as assemble<T,true>).
template <typename T>
__device__ __forceinline__ void assemble_fast(const Frozen<T>& F, T ul, T ur, T vt, T vb, T Hc, T fu_l, T fu_r,
                                              T fv_t, T fv_b, T fH, T thk, T dti, const Phys<T>& p, T (&J)[25],
                                              T (&r)[5]) {
    const T dxi = p.dxi;
    const T gc = sigmoid(F.bed_c + rho_ratio<T>() * Hc, p.sig_c);
    // mass row
    {
        Calving<T> cv = calving_g(Hc, gc, p);
        Flux<T> ql = upwind_flux(ul, F.H_l, Hc, F.w_l > T(0));
        Flux<T> qr = upwind_flux(ur, Hc, F.H_r, F.w_r > T(0));
        Flux<T> qt = upwind_flux(vt, Hc, F.H_t, F.w_t > T(0));
        Flux<T> qb = upwind_flux(vb, F.H_b, Hc, F.w_b > T(0));
        T r4 = Hc * dti - fH - cv.res - ql.res * dxi + qr.res * dxi + qt.res * dxi - qb.res * dxi;
        if ((Hc - p.dt * r4) <= thk) {
            J[20] = T(0); J[21] = T(0); J[22] = T(0); J[23] = T(0); J[24] = T(1);
            r[4] = Hc - thk;
        } else {
            J[20] = -ql.d_vel * dxi;
            J[21] = qr.d_vel * dxi;
            J[22] = qt.d_vel * dxi;
            J[23] = -qb.d_vel * dxi;
            J[24] = dti - cv.d_H + (-ql.d_Hb + qr.d_Ha + qt.d_Ha - qb.d_Hb) * dxi;
            r[4] = r4;
        }
    }
    // own-cell normal stresses
    const T etaH = F.eta_c * Hc;
    const T pre = T(2) * etaH * dxi;
    const T exx = T(2) * (ur - ul) * dxi + (vt - vb) * dxi;
    const T eyy = (ur - ul) * dxi + T(2) * (vt - vb) * dxi;
    const T sxx = T(2) * etaH * exx, syy = T(2) * etaH * eyy;
    const T hx = T(2) * exx * F.eta_c * dxi, hy = T(2) * eyy * F.eta_c * dxi;
    const T p2 = pre * dxi;
    J[0] = -T(2) * p2; J[1] = T(2) * p2; J[2] = p2; J[3] = -p2; J[4] = hx;
    J[5] = T(2) * p2; J[6] = -T(2) * p2; J[7] = -p2; J[8] = p2; J[9] = -hx;
    J[10] = p2; J[11] = -p2; J[12] = -T(2) * p2; J[13] = T(2) * p2; J[14] = -hy;
    J[15] = -p2; J[16] = p2; J[17] = T(2) * p2; J[18] = -T(2) * p2; J[19] = hy;
    T r0 = -fu_l + sxx * dxi, r1 = -fu_r - sxx * dxi, r2 = -fv_t - syy * dxi, r3 = -fv_b + syy * dxi;
    // neighbour normal stresses
    r0 -= (F.kl * (ul - F.u_ll) + F.cl) * dxi;   J[0] -= F.kl * dxi;
    r1 += (F.kr * (F.u_rr - ur) + F.cr) * dxi;   J[6] -= F.kr * dxi;
    r2 += (F.kt * (F.v_tt - vt) + F.ct) * dxi;   J[12] -= F.kt * dxi;
    r3 -= (F.kb * (vb - F.v_bb) + F.cb) * dxi;   J[18] -= F.kb * dxi;
    // corner shear stresses
    {
        const T ecH = F.ec * Hc;
        T eH = (F.S_tl + ecH) * F.w_tl;
        T exy = T(0.5) * ((F.u_tl - ul) * dxi + (vt - F.v_lt) * dxi);
        T res = T(2) * eH * exy * dxi, dd = eH * dxi * dxi, de = T(2) * exy * F.w_tl * F.ec * dxi;
        r0 += res; r2 -= res; J[0] -= dd; J[4] += de; J[12] -= dd; J[14] -= de;
        eH = (F.S_tr + ecH) * F.w_tr;
        exy = T(0.5) * ((F.u_tr - ur) * dxi + (F.v_rt - vt) * dxi);
        res = T(2) * eH * exy * dxi; dd = eH * dxi * dxi; de = T(2) * exy * F.w_tr * F.ec * dxi;
        r1 += res; r2 += res; J[6] -= dd; J[9] += de; J[12] -= dd; J[14] += de;
        eH = (F.S_bl + ecH) * F.w_bl;
        exy = T(0.5) * ((ul - F.u_bl) * dxi + (vb - F.v_lb) * dxi);
        res = T(2) * eH * exy * dxi; dd = eH * dxi * dxi; de = T(2) * exy * F.w_bl * F.ec * dxi;
        r0 -= res; r3 -= res; J[0] -= dd; J[4] -= de; J[18] -= dd; J[19] -= de;
        eH = (F.S_br + ecH) * F.w_br;
        exy = T(0.5) * ((ur - F.u_br) * dxi + (F.v_rb - vb) * dxi);
        res = T(2) * eH * exy * dxi; dd = eH * dxi * dxi; de = T(2) * exy * F.w_br * F.ec * dxi;
        r1 -= res; r3 += res; J[6] -= dd; J[9] -= de; J[18] -= dd; J[19] += de;
    }
    // basal drag
    {
        const T bec = gc * F.beta_c + (T(1) - gc) * p.water_drag;
        T bl = T(0.5) * (F.be_l + bec), br = T(0.5) * (bec + F.be_r);
        T bt = T(0.5) * (F.be_t + bec), bb = T(0.5) * (bec + F.be_b);
        r0 -= bl * ul; r1 -= br * ur; r2 -= bt * vt; r3 -= bb * vb;
        J[0] -= bl; J[6] -= br; J[12] -= bt; J[18] -= bb;
        if (p.gl_deriv) {
            T dgc = rho_ratio<T>() * (p.sig_c * gc * (T(1) - gc)) * (F.beta_c - p.water_drag);
            J[4] += T(-0.5) * dgc * ul;
            J[9] += T(-0.5) * dgc * ur;
            J[14] += T(-0.5) * dgc * vt;
            J[19] += T(-0.5) * dgc * vb;
        }
    }
    // driving stress; x: left (m) / right (p); y: bottom (m) / top (p)
    {
        const T bc = M<T>::max(F.bed_c, -rho_ratio<T>() * Hc);
        const T Sc = bc + Hc;
        const T dbc = T(1) + (F.bed_c > -rho_ratio<T>() * Hc ? T(0) : -rho_ratio<T>());
        // left face: m = left, p = this cell
        T Havg = T(0.5) * (F.H_l + Hc), dS = Sc - F.S_l;
        r0 -= Havg * dS * dxi * F.w_l;
        J[4] -= (T(0.5) * dS * dxi + Havg * dbc * dxi) * F.w_l;
        // right face: m = this cell, p = right
        Havg = T(0.5) * (Hc + F.H_r); dS = F.S_r - Sc;
        r1 -= Havg * dS * dxi * F.w_r;
        J[9] -= (T(0.5) * dS * dxi - Havg * dbc * dxi) * F.w_r;
        // top face: m = this cell (bottom), p = top
        Havg = T(0.5) * (Hc + F.H_t); dS = F.S_t - Sc;
        r2 -= Havg * dS * dxi * F.w_t;
        J[14] -= (T(0.5) * dS * dxi - Havg * dbc * dxi) * F.w_t;
        // bottom face: m = bottom, p = this cell (top)
        Havg = T(0.5) * (F.H_b + Hc); dS = Sc - F.S_b;
        r3 -= Havg * dS * dxi * F.w_b;
        J[19] -= (T(0.5) * dS * dxi + Havg * dbc * dxi) * F.w_b;
    }
    r[0] = r0; r[1] = r1; r[2] = r2; r[3] = r3;
}

// LU solve with the pivot reciprocals reused in the back substitution.
template <typename T> __device__ __forceinline__ void lu5_solve_fast(T (&A)[25], const T (&b)[5], T (&x)[5]) {
    T inv[5];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        inv[k] = M<T>::rcp(A[k * 5 + k]);
#pragma unroll
        for (int i = k + 1; i < 5; i++) {
            A[i * 5 + k] *= inv[k];
#pragma unroll
            for (int j = k + 1; j < 5; j++) A[i * 5 + j] -= A[i * 5 + k] * A[k * 5 + j];
        }
    }
    T y1 = b[1] - A[5] * b[0];
    T y2 = b[2] - A[10] * b[0] - A[11] * y1;
    T y3 = b[3] - A[15] * b[0] - A[16] * y1 - A[17] * y2;
    T y4 = b[4] - A[20] * b[0] - A[21] * y1 - A[22] * y2 - A[23] * y3;
    x[4] = y4 * inv[4];
    x[3] = (y3 - A[19] * x[4]) * inv[3];
    x[2] = (y2 - A[13] * x[3] - A[14] * x[4]) * inv[2];
    x[1] = (y1 - A[7] * x[2] - A[8] * x[3] - A[9] * x[4]) * inv[1];
    x[0] = (b[0] - A[1] * x[1] - A[2] * x[2] - A[3] * x[3] - A[4] * x[4]) * inv[0];
}

// 5x5 solve with partial (row) pivoting, the robustness variant of the
// reference (lu_5x5_solve_pivot, glide/cuda/common.cu:180-233): the largest
// |entry| of the column becomes the pivot (first one on ties), a pivot below
// 1e-14 in magnitude skips its elimination step, a diagonal below 1e-14 in
// back substitution gives x = 0.  Rows are swapped in registers by unrolled
// conditional moves.
template <typename T> __device__ __forceinline__ void lu5_solve_pivot(T (&A)[25], const T (&b)[5], T (&x)[5]) {
    T y[5] = {b[0], b[1], b[2], b[3], b[4]};
    const T tiny = T(1e-14);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        int p = k;
        T best = M<T>::abs(A[k * 5 + k]);
#pragma unroll
        for (int i = k + 1; i < 5; i++) {
            const T a = M<T>::abs(A[i * 5 + k]);
            if (a > best) {
                best = a;
                p = i;
            }
        }
#pragma unroll
        for (int i = k + 1; i < 5; i++) {
            if (i == p) {
#pragma unroll
                for (int j = 0; j < 5; j++) {
                    const T t = A[k * 5 + j];
                    A[k * 5 + j] = A[i * 5 + j];
                    A[i * 5 + j] = t;
                }
                const T t = y[k];
                y[k] = y[i];
                y[i] = t;
            }
        }
        const T piv = A[k * 5 + k];
        if (M<T>::abs(piv) < tiny) continue;
#pragma unroll
        for (int i = k + 1; i < 5; i++) {
            const T f = A[i * 5 + k] / piv;
            A[i * 5 + k] = f;
#pragma unroll
            for (int j = k + 1; j < 5; j++) A[i * 5 + j] -= f * A[k * 5 + j];
        }
    }
#pragma unroll
    for (int i = 1; i < 5; i++) {
#pragma unroll
        for (int j = 0; j < i; j++) y[i] -= A[i * 5 + j] * y[j];
    }
#pragma unroll
    for (int i = 4; i >= 0; i--) {
        T v = y[i];
#pragma unroll
        for (int j = i + 1; j < 5; j++) v -= A[i * 5 + j] * x[j];
        const T d = A[i * 5 + i];
        x[i] = M<T>::abs(d) > tiny ? v / d : T(0);
    }
}

// Per-cell Newton deltas.  scratch holds 5 cell arrays: 0.5*du_l, 0.5*du_r,
// 0.5*dv_t, 0.5*dv_b, dH.
template <typename T, bool LOCAL>
#ifndef GLIDE_VANKA64_MIN_BLOCKS
#define GLIDE_VANKA64_MIN_BLOCKS 2
#endif
#ifndef GLIDE_VANKA32_MIN_BLOCKS
#define GLIDE_VANKA32_MIN_BLOCKS 2
#endif
__global__ void __launch_bounds__(VNT, sizeof(T) == 4 ? GLIDE_VANKA32_MIN_BLOCKS : GLIDE_VANKA64_MIN_BLOCKS) vanka_cells_kernel(
    T* __restrict__ scratch, const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ f_u, const T* __restrict__ f_v, const T* __restrict__ f_H, const T* __restrict__ bed,
    const T* __restrict__ B, const T* __restrict__ beta, const T* __restrict__ gamma, const int* __restrict__ flags,
    const int* __restrict__ any_active, int n_newton, T shift, T step, int pivot, Geo g, Phys<T> p) {
    __shared__ T s_eta[VY + 2][VX + 2];
    const int ny = g.ny, nx = g.nx;
    const int bz = blockIdx.z;
    if (LOCAL && any_active[bz] == 0) return;
    u += bz * g.nu(); v += bz * g.nv(); H += bz * g.nc(); f_u += bz * g.nu(); f_v += bz * g.nv();
    f_H += bz * g.nc(); bed += bz * g.nc(); B += bz * g.nc(); beta += bz * g.nc(); gamma += bz * g.nc();
    const int64_t nc = g.nc();
    scratch += bz * 5 * nc;
    if (LOCAL) flags += bz * int64_t(ny / REF_STRIDE + 1) * (nx / REF_STRIDE + 1);
    const int i0 = blockIdx.y * VY, j0 = blockIdx.x * VX;
    const int r = threadIdx.x / VX, c = threadIdx.x % VX;
    const int i = i0 + r, j = j0 + c;
    eta_window(s_eta, u, v, B, i0, j0, ny, nx, p);
    __syncthreads();
    if (i >= ny || j >= nx) return;
    if (LOCAL && !ref_tile_on(flags, i, j, nx)) return;

    Frozen<T> F;
    {
        Patch<T> P;
        load_patch(P, s_eta, r, c, u, v, H, bed, beta, i, j, ny, nx, p);
        make_frozen(F, P, ny, nx, p);
    }
    // 32-bit offsets within one field (the entry points bound a field below 2^31 elements)
    const int iu = i * (nx + 1) + j, ic32 = i * nx + j;
    const T ul0 = u[iu], ur0 = u[iu + 1];
    const T vt0 = v[ic32], vb0 = v[ic32 + nx];
    const T H0 = H[ic32];
    const T fu_l = f_u[iu], fu_r = f_u[iu + 1];
    const T fv_t = f_v[ic32], fv_b = f_v[ic32 + nx];
    const T fH = f_H[ic32];
    const T thk = gamma[ic32];
    const T dti = T(1) / p.dt;
    T ul = ul0, ur = ur0, vt = vt0, vb = vb0, Hc = H0;
    for (int it = 0; it < n_newton; it++) {
        T J[25], rr[5], x[5];
        assemble_fast<T>(F, ul, ur, vt, vb, Hc, fu_l, fu_r, fv_t, fv_b, fH, thk, dti, p, J, rr);
        J[0] -= shift; J[6] -= shift; J[12] -= shift; J[18] -= shift; J[24] += shift;  // vanka.cu:406-410
        if (pivot)
            lu5_solve_pivot(J, rr, x);
        else
            lu5_solve_fast(J, rr, x);
        ul -= step * x[0];  // reference step 0.25: relaxation_factor, glide/cuda/vanka.cu:416
        ur -= step * x[1];
        vt -= step * x[2];
        vb -= step * x[3];
        Hc -= step * x[4];
        Hc = M<T>::max(Hc, thk);
    }
    if (!(isfinite(ul) && isfinite(ur) && isfinite(vt) && isfinite(vb) && isfinite(Hc))) {
        ul = ul0, ur = ur0, vt = vt0, vb = vb0, Hc = H0;  // a failed local solve leaves its cell unchanged
    }
    const int64_t ic = int64_t(i) * nx + j;
    scratch[ic] = T(0.5) * (ul - ul0);
    scratch[nc + ic] = T(0.5) * (ur - ur0);
    scratch[2 * nc + ic] = T(0.5) * (vt - vt0);
    scratch[3 * nc + ic] = T(0.5) * (vb - vb0);
    scratch[4 * nc + ic] = Hc - H0;
}

// --------------------------------------------------------------------------
// Linear Vanka for defect correction (no counterpart in the reference): the
// local 5x5 matrix of each cell at the current state (the same matrix the
// first Newton iteration of vanka_cells_kernel factors) is factored once and
// stored; each sweep then solves it against the cell's part of the linear
// residual rho = r + J d, giving the additive-Vanka update of the correction
// d with the H >= gamma bound applied to H + d_H.
// --------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void lu5_factor(T (&A)[25]) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const T inv = M<T>::rcp(A[k * 5 + k]);
#pragma unroll
        for (int i = k + 1; i < 5; i++) {
            A[i * 5 + k] *= inv;
#pragma unroll
            for (int j = k + 1; j < 5; j++) A[i * 5 + j] -= A[i * 5 + k] * A[k * 5 + j];
        }
        A[k * 5 + k] = inv;  // stored as the reciprocal pivot
    }
}
template <typename T>
__device__ __forceinline__ void lu5_subst(const T (&A)[25], const T (&b)[5], T (&x)[5]) {
    T y1 = b[1] - A[5] * b[0];
    T y2 = b[2] - A[10] * b[0] - A[11] * y1;
    T y3 = b[3] - A[15] * b[0] - A[16] * y1 - A[17] * y2;
    T y4 = b[4] - A[20] * b[0] - A[21] * y1 - A[22] * y2 - A[23] * y3;
    x[4] = y4 * A[24];
    x[3] = (y3 - A[19] * x[4]) * A[18];
    x[2] = (y2 - A[13] * x[3] - A[14] * x[4]) * A[12];
    x[1] = (y1 - A[7] * x[2] - A[8] * x[3] - A[9] * x[4]) * A[6];
    x[0] = (b[0] - A[1] * x[1] - A[2] * x[2] - A[3] * x[3] - A[4] * x[4]) * A[0];
}

// lu[k * nc + cell], k = 0..24: factors of the cell's local matrix at U.
template <typename T>
__global__ void __launch_bounds__(VNT, sizeof(T) == 4 ? 2 : GLIDE_VANKA64_MIN_BLOCKS) vanka_lu_kernel(
    T* __restrict__ lu, const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ f_H, const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta,
    const T* __restrict__ gamma, const T* __restrict__ act, T shift, Geo g, Phys<T> p) {
    __shared__ T s_eta[VY + 2][VX + 2];
    const int ny = g.ny, nx = g.nx;
    const int bz = blockIdx.z;
    u += bz * g.nu(); v += bz * g.nv(); H += bz * g.nc();
    if (act) act += bz * g.nc(); else f_H += bz * g.nc();
    bed += bz * g.nc(); B += bz * g.nc(); beta += bz * g.nc(); gamma += bz * g.nc();
    const int64_t nc = g.nc();
    lu += bz * 25 * nc;
    const int i0 = blockIdx.y * VY, j0 = blockIdx.x * VX;
    const int r = threadIdx.x / VX, c = threadIdx.x % VX;
    const int i = i0 + r, j = j0 + c;
    eta_window(s_eta, u, v, B, i0, j0, ny, nx, p);
    __syncthreads();
    if (i >= ny || j >= nx) return;
    Frozen<T> F;
    {
        Patch<T> P;
        load_patch(P, s_eta, r, c, u, v, H, bed, beta, i, j, ny, nx, p);
        make_frozen(F, P, ny, nx, p);
    }
    const int64_t ic = int64_t(i) * nx + j;
    const T ul = u[int64_t(i) * (nx + 1) + j], ur = u[int64_t(i) * (nx + 1) + j + 1];
    const T vt = v[ic], vb = v[int64_t(i + 1) * nx + j];
    T J[25], rr[5];
    // the momentum rows do not depend on f; the mass row's active-set switch
    // (vanka.cu:104-113) needs the local mass residual, hence f_H.  With a
    // given active set (act) the switch is forced instead: a right-hand side
    // of -/+1e30 makes H - dt r_H far below / above gamma (r is discarded).
    const T fH = act ? (act[ic] > T(0.5) ? T(-1e30) : T(1e30)) : f_H[ic];
    assemble_fast<T>(F, ul, ur, vt, vb, H[ic], T(0), T(0), T(0), T(0), fH, gamma[ic], T(1) / p.dt, p, J, rr);
    J[0] -= shift; J[6] -= shift; J[12] -= shift; J[18] -= shift; J[24] += shift;  // vanka.cu:406-410
    lu5_factor(J);
#pragma unroll
    for (int k = 0; k < 25; k++) lu[k * nc + ic] = J[k];
}

// scratch = the additive-Vanka halves of -A^-1 rho (same layout as
// vanka_cells_kernel), with H + d_H + delta_H >= gamma.
template <typename T>
__global__ void vanka_linear_kernel(T* __restrict__ scratch, const T* __restrict__ lu,
                                    const T* __restrict__ rho_u, const T* __restrict__ rho_v,
                                    const T* __restrict__ rho_H, const T* __restrict__ H,
                                    const T* __restrict__ dH, const T* __restrict__ gamma, Geo g) {
    const int ny = g.ny, nx = g.nx;
    const int bz = blockIdx.z;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= ny || j >= nx) return;
    const int64_t nc = g.nc();
    rho_u += bz * g.nu(); rho_v += bz * g.nv(); rho_H += bz * nc; H += bz * nc; dH += bz * nc;
    gamma += bz * nc; lu += bz * 25 * nc; scratch += bz * 5 * nc;
    const int64_t ic = int64_t(i) * nx + j;
    T A[25];
#pragma unroll
    for (int k = 0; k < 25; k++) A[k] = lu[k * nc + ic];
    const T b[5] = {rho_u[int64_t(i) * (nx + 1) + j], rho_u[int64_t(i) * (nx + 1) + j + 1], rho_v[ic],
                    rho_v[int64_t(i + 1) * nx + j], rho_H[ic]};
    T x[5];
    lu5_subst(A, b, x);
    T dHc = -x[4];
    dHc = M<T>::max(dHc, gamma[ic] - H[ic] - dH[ic]);
    if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]) && isfinite(x[3]) && isfinite(dHc))) {
        x[0] = x[1] = x[2] = x[3] = T(0);
        dHc = T(0);
    }
    scratch[ic] = T(-0.5) * x[0];
    scratch[nc + ic] = T(-0.5) * x[1];
    scratch[2 * nc + ic] = T(-0.5) * x[2];
    scratch[3 * nc + ic] = T(-0.5) * x[3];
    scratch[4 * nc + ic] = dHc;
}

// U += omega * delta, face delta = sum of the two adjacent cells' halves.
template <typename T, bool LOCAL>
__global__ void vanka_apply_kernel(T* __restrict__ u, T* __restrict__ v, T* __restrict__ H,
                                   const T* __restrict__ scratch, const int* __restrict__ flags,
                                   const int* __restrict__ any_active, T omega, Geo g) {
    const int ny = g.ny, nx = g.nx;
    const int bz = blockIdx.z;
    if (LOCAL && any_active[bz] == 0) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i > ny || j > nx) return;
    const int64_t nc = g.nc();
    u += bz * g.nu(); v += bz * g.nv(); H += bz * g.nc();
    scratch += bz * 5 * nc;
    if (LOCAL) flags += bz * int64_t(ny / REF_STRIDE + 1) * (nx / REF_STRIDE + 1);
    auto on = [&](int ii, int jj) { return !LOCAL || ref_tile_on(flags, ii, jj, nx); };
    if (i < ny) {  // u-face (i,j), j in [0,nx]
        T d = T(0);
        if (j < nx && on(i, j)) d += scratch[int64_t(i) * nx + j];                   // as u_l of cell (i,j)
        if (j > 0 && on(i, j - 1)) d += scratch[nc + int64_t(i) * nx + j - 1];        // as u_r of cell (i,j-1)
        u[int64_t(i) * (nx + 1) + j] += omega * d;
    }
    if (j < nx) {  // v-face (i,j), i in [0,ny]
        T d = T(0);
        if (i < ny && on(i, j)) d += scratch[2 * nc + int64_t(i) * nx + j];
        if (i > 0 && on(i - 1, j)) d += scratch[3 * nc + int64_t(i - 1) * nx + j];
        v[int64_t(i) * nx + j] += omega * d;
    }
    if (i < ny && j < nx && on(i, j)) H[int64_t(i) * nx + j] += omega * scratch[4 * nc + int64_t(i) * nx + j];
}

// Local error indicator (glide/solver.py:148-154) and reference-tile flags.
// err = |r_u(l)| + |r_u(r)| + |r_v(t)| + |r_v(b)| + |FB(r_H, H-gamma)| > threshold
template <typename T>
__global__ void error_mask_kernel(T* __restrict__ err_mask, const T* __restrict__ r_u, const T* __restrict__ r_v,
                                  const T* __restrict__ r_H, const T* __restrict__ H, const T* __restrict__ gamma,
                                  T threshold, Geo g) {
    const int ny = g.ny, nx = g.nx;
    const int bz = blockIdx.z;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= ny || j >= nx) return;
    r_u += bz * g.nu(); r_v += bz * g.nv(); r_H += bz * g.nc(); H += bz * g.nc(); gamma += bz * g.nc();
    err_mask += bz * g.nc();
    const int64_t ic = int64_t(i) * nx + j;
    T a = r_H[ic], b = H[ic] - gamma[ic];
    T fb = a + b - M<T>::sqrt(a * a + b * b);
    T tot = M<T>::abs(r_u[int64_t(i) * (nx + 1) + j + 1]) + M<T>::abs(r_u[int64_t(i) * (nx + 1) + j]) +
            M<T>::abs(r_v[int64_t(i + 1) * nx + j]) + M<T>::abs(r_v[ic]) + M<T>::abs(fb);
    err_mask[ic] = tot > threshold ? T(1) : T(0);
}

// One CTA per reference block: flag = any in-domain cell of the 16x16 window
// has err_mask > 0.5.  any_active[b] counts active blocks.
template <typename T>
__global__ void tile_flags_kernel(int* __restrict__ flags, int* __restrict__ any_active,
                                  const T* __restrict__ err_mask, Geo g) {
    const int ny = g.ny, nx = g.nx;
    const int bz = blockIdx.z;
    const int nbx = nx / REF_STRIDE + 1;
    const int bx = blockIdx.x, by = blockIdx.y;
    err_mask += bz * g.nc();
    flags += bz * int64_t(ny / REF_STRIDE + 1) * nbx;
    const int i = by * REF_STRIDE - 1 + threadIdx.y;
    const int j = bx * REF_STRIDE - 1 + threadIdx.x;
    bool bad = (i >= 0 && i < ny && j >= 0 && j < nx) && err_mask[int64_t(i) * nx + j] > T(0.5);
    int any = __syncthreads_or(bad);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        flags[by * nbx + bx] = any;
        if (any) atomicAdd(any_active + bz, 1);
    }
}

// --------------------------------------------------------------------------
// adjoint Vanka, one colour (glide/cuda/vanka.cu:441-840)
// Solves J^T dlam = r_adj per cell of the colour with the local Jacobian at
// the current state (mask>0.5 rows replaced by the identity, no shift) and
// updates lambda in place: each face is adjacent to exactly one cell of a
// colour, so every lambda entry has a single writer.
// --------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(VNT) vanka_adjoint_kernel(
    T* __restrict__ lu, T* __restrict__ lv, T* __restrict__ lH, const T* __restrict__ ra_u,
    const T* __restrict__ ra_v, const T* __restrict__ ra_H, const T* __restrict__ u, const T* __restrict__ v,
    const T* __restrict__ H, const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta,
    const T* __restrict__ mask, int color, T omega, Geo g, Phys<T> p) {
    __shared__ T s_eta[VY + 2][VX + 2];
    const int ny = g.ny, nx = g.nx;
    const int bz = blockIdx.z;
    u += bz * g.nu(); v += bz * g.nv(); H += bz * g.nc(); bed += bz * g.nc(); B += bz * g.nc();
    beta += bz * g.nc(); mask += bz * g.nc(); lu += bz * g.nu(); lv += bz * g.nv(); lH += bz * g.nc();
    ra_u += bz * g.nu(); ra_v += bz * g.nv(); ra_H += bz * g.nc();
    const int i0 = blockIdx.y * VY, j0 = blockIdx.x * VX;
    const int r = threadIdx.x / VX, c = threadIdx.x % VX;
    const int i = i0 + r, j = j0 + c;
    eta_window(s_eta, u, v, B, i0, j0, ny, nx, p);
    __syncthreads();
    if (i >= ny || j >= nx || ((i + j) & 1) != color) return;
    Patch<T> P;
    load_patch(P, s_eta, r, c, u, v, H, bed, beta, i, j, ny, nx, p);
    const int64_t iu = int64_t(i) * (nx + 1) + j, ic = int64_t(i) * nx + j, ivb = int64_t(i + 1) * nx + j;
    T J[25], rr[5];
    assemble<T, false>(P, u[iu], u[iu + 1], v[ic], v[ivb], H[ic], T(0), T(0), T(0), T(0), T(0), T(0), ny, nx, p,
                       J, rr);
    if (mask[ic] > T(0.5)) {
        J[20] = T(0); J[21] = T(0); J[22] = T(0); J[23] = T(0); J[24] = T(1);
    }
    T JT[25];
#pragma unroll
    for (int a = 0; a < 5; a++)
#pragma unroll
        for (int b = 0; b < 5; b++) JT[a * 5 + b] = J[b * 5 + a];
    T rhs[5] = {ra_u[iu], ra_u[iu + 1], ra_v[ic], ra_v[ivb], ra_H[ic]};
    T x[5];
    lu5_solve(JT, rhs, x);
    lu[iu] += T(0.5) * omega * x[0];
    lu[iu + 1] += T(0.5) * omega * x[1];
    lv[ic] += T(0.5) * omega * x[2];
    lv[ivb] += T(0.5) * omega * x[3];
    lH[ic] += omega * x[4];
}

// --------------------------------------------------------------------------
// launchers
// --------------------------------------------------------------------------
static inline dim3 cell_grid(const Geo& g) { return dim3((g.nx + VX - 1) / VX, (g.ny + VY - 1) / VY, g.nb); }
static inline dim3 face_grid(const Geo& g) { return dim3((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, g.nb); }

template <typename T>
int launch_vanka_sweeps(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_iter,
                        int n_newton, double omega, double shift, const int* flags, const int* any_active,
                        void* scratch, cudaStream_t s, double newton_step, int pivot) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    T* u = (T*)a->u;
    T* v = (T*)a->v;
    T* H = (T*)a->H;
    for (int k = 0; k < n_iter; k++) {
        if (flags) {
            glide::count_launch(), vanka_cells_kernel<T, true><<<cell_grid(g), VNT, 0, s>>>(
                (T*)scratch, u, v, H, (const T*)f_u, (const T*)f_v, (const T*)f_H, (const T*)a->bed,
                (const T*)a->B, (const T*)a->beta, (const T*)a->gamma, flags, any_active, n_newton, T(shift), T(newton_step), pivot, g, p);
            glide::count_launch(), vanka_apply_kernel<T, true><<<face_grid(g), dim3(32, 8), 0, s>>>(u, v, H, (const T*)scratch, flags,
                                                                               any_active, T(omega), g);
        } else {
            glide::count_launch(), vanka_cells_kernel<T, false><<<cell_grid(g), VNT, 0, s>>>(
                (T*)scratch, u, v, H, (const T*)f_u, (const T*)f_v, (const T*)f_H, (const T*)a->bed,
                (const T*)a->B, (const T*)a->beta, (const T*)a->gamma, nullptr, nullptr, n_newton, T(shift), T(newton_step), pivot, g, p);
            glide::count_launch(), vanka_apply_kernel<T, false><<<face_grid(g), dim3(32, 8), 0, s>>>(u, v, H, (const T*)scratch, nullptr,
                                                                                nullptr, T(omega), g);
        }
    }
    return (int)cudaGetLastError();
}

// Only the per-cell Newton kernel, n_launch times (profiling / timing; U is not updated).
template <typename T>
int launch_vanka_cells(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_launch,
                       int n_newton, double shift, const int* flags, const int* any_active, void* scratch,
                       cudaStream_t s, double newton_step) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    for (int k = 0; k < n_launch; k++) {
        if (flags)
            glide::count_launch(), vanka_cells_kernel<T, true><<<cell_grid(g), VNT, 0, s>>>(
                (T*)scratch, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)f_u, (const T*)f_v,
                (const T*)f_H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->gamma, flags,
                any_active, n_newton, T(shift), T(newton_step), 0, g, p);
        else
            glide::count_launch(), vanka_cells_kernel<T, false><<<cell_grid(g), VNT, 0, s>>>(
                (T*)scratch, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)f_u, (const T*)f_v,
                (const T*)f_H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->gamma, nullptr,
                nullptr, n_newton, T(shift), T(newton_step), 0, g, p);
    }
    return (int)cudaGetLastError();
}

template <typename T>
int launch_vanka_lu(const GlideLevelArgs* a, const void* f_H, void* lu, double shift, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    // f_H null: the active set is the level's mask (glide_vanka_lu_masked)
    glide::count_launch(), vanka_lu_kernel<T><<<cell_grid(g), VNT, 0, s>>>(
        (T*)lu, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)f_H, (const T*)a->bed, (const T*)a->B,
        (const T*)a->beta, (const T*)a->gamma, f_H ? nullptr : (const T*)a->mask, T(shift), g, p);
    return (int)cudaGetLastError();
}

// d += omega * (linear Vanka update of rho), n_iter times with a fixed rho is
// not useful: one sweep per call, rho recomputed by the caller in between.
template <typename T>
int launch_vanka_linear(const GlideLevelArgs* a, const void* rho_u, const void* rho_v, const void* rho_H,
                        const void* lu, void* d_u, void* d_v, void* d_H, double omega, void* scratch,
                        cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    dim3 blk(32, 8);
    dim3 grd((g.nx + 31) / 32, (g.ny + 7) / 8, g.nb);
    glide::count_launch(), vanka_linear_kernel<T><<<grd, blk, 0, s>>>(
        (T*)scratch, (const T*)lu, (const T*)rho_u, (const T*)rho_v, (const T*)rho_H, (const T*)a->H,
        (const T*)d_H, (const T*)a->gamma, g);
    glide::count_launch(), vanka_apply_kernel<T, false><<<face_grid(g), dim3(32, 8), 0, s>>>(
        (T*)d_u, (T*)d_v, (T*)d_H, (const T*)scratch, nullptr, nullptr, T(omega), g);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_error_mask(const GlideLevelArgs* a, const void* r_u, const void* r_v, const void* r_H, double threshold,
                      void* err_mask, int* flags, int* any_active, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    dim3 blk(32, 8);
    dim3 grd((g.nx + 31) / 32, (g.ny + 7) / 8, g.nb);
    glide::count_launch(), error_mask_kernel<T><<<grd, blk, 0, s>>>((T*)err_mask, (const T*)r_u, (const T*)r_v, (const T*)r_H,
                                             (const T*)a->H, (const T*)a->gamma, T(threshold), g);
    if (flags) {
        cudaMemsetAsync(any_active, 0, sizeof(int) * g.nb, s);
        dim3 tg(g.nx / REF_STRIDE + 1, g.ny / REF_STRIDE + 1, g.nb);
        glide::count_launch(), tile_flags_kernel<T><<<tg, dim3(REF_WIN, REF_WIN), 0, s>>>(flags, any_active, (const T*)err_mask, g);
    }
    return (int)cudaGetLastError();
}

template <typename T>
int launch_tile_flags(const GlideLevelArgs* a, const void* err_mask, int* flags, int* any_active, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    cudaMemsetAsync(any_active, 0, sizeof(int) * g.nb, s);
    dim3 tg(g.nx / REF_STRIDE + 1, g.ny / REF_STRIDE + 1, g.nb);
    glide::count_launch(), tile_flags_kernel<T><<<tg, dim3(REF_WIN, REF_WIN), 0, s>>>(flags, any_active, (const T*)err_mask, g);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_vanka_adjoint(const GlideLevelArgs* a, void* l_u, void* l_v, void* l_H, const void* ra_u, const void* ra_v,
                         const void* ra_H, int color, double omega, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    glide::count_launch(), vanka_adjoint_kernel<T><<<cell_grid(g), VNT, 0, s>>>(
        (T*)l_u, (T*)l_v, (T*)l_H, (const T*)ra_u, (const T*)ra_v, (const T*)ra_H, (const T*)a->u, (const T*)a->v,
        (const T*)a->H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->mask, color, T(omega), g,
        p);
    return (int)cudaGetLastError();
}

#define INST(T)                                                                                                  \
    template int launch_vanka_sweeps<T>(const GlideLevelArgs*, const void*, const void*, const void*, int, int,   \
                                        double, double, const int*, const int*, void*, cudaStream_t, double, int);\
    template int launch_vanka_cells<T>(const GlideLevelArgs*, const void*, const void*, const void*, int, int,     \
                                       double, const int*, const int*, void*, cudaStream_t, double);              \
    template int launch_error_mask<T>(const GlideLevelArgs*, const void*, const void*, const void*, double,       \
                                      void*, int*, int*, cudaStream_t);                                           \
    template int launch_tile_flags<T>(const GlideLevelArgs*, const void*, int*, int*, cudaStream_t);              \
    template int launch_vanka_adjoint<T>(const GlideLevelArgs*, void*, void*, void*, const void*, const void*,    \
                                         const void*, int, double, cudaStream_t);                                 \
    template int launch_vanka_lu<T>(const GlideLevelArgs*, const void*, void*, double, cudaStream_t);             \
    template int launch_vanka_linear<T>(const GlideLevelArgs*, const void*, const void*, const void*, const void*, \
                                        void*, void*, void*, double, void*, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace glide
