// Residual, JVP, VJP and basal-friction gradient kernels for the SSA system
// on the MAC staggered grid.
//
// Structure (B200): a CTA owns a 32x16 tile of cells with the u-faces on
// their left, the v-faces on their top (plus the closing face row/column at
// the domain edge).  Phase 1 computes the cell viscosity (and its tangent) for
// the tile plus a one-cell ring into shared memory; phase 2 turns it into
// the cell normal stresses and vertex shear stresses the tile needs; phase 3
// writes each owned residual entry as a divergence of those stresses plus
// the face-local drag/driving terms.  Every output has exactly one writer,
// so results are deterministic (the reference scatters with float atomics,
// glide/cuda/residuals.cu:617-1021).
#include "glide_common.cuh"

namespace glide {

constexpr int TX = 32;               // tile columns (one warp across)
constexpr int NTHR = 256;            // threads per CTA (32 x 8)
constexpr int WC = TX + 2;           // window columns (one-cell ring)

struct TileIdx {
    int i0, j0, tx, ty, tid;
};
template <int TYK> __device__ __forceinline__ TileIdx tile_idx() {
    TileIdx t;
    t.tx = threadIdx.x % TX;
    t.ty = threadIdx.x / TX;
    t.tid = threadIdx.x;
    t.i0 = blockIdx.y * TYK;
    t.j0 = blockIdx.x * TX;
    return t;
}

// --------------------------------------------------------------------------
// residual r = F(U) - f with the active-set row, or the JVP J(U) d
// (glide/cuda/residuals.cu:6-579)
// --------------------------------------------------------------------------
constexpr int TY = 16;                 // residual/JVP tile rows
constexpr int RPT = TY / (NTHR / TX);  // rows per thread = 2
constexpr int WR = TY + 2;

template <typename T, bool TAN>
__global__ void __launch_bounds__(NTHR) stencil_kernel(
    T* __restrict__ o_u, T* __restrict__ o_v, T* __restrict__ o_H,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ a_u, const T* __restrict__ a_v, const T* __restrict__ a_H,  // f (residual) or d (JVP)
    const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta,
    const T* __restrict__ mask, const T* __restrict__ gamma, Geo g, Phys<T> p) {
    __shared__ T s_etaH[WR][WC];
    __shared__ T s_eta[WR][WC];
    __shared__ T s_sxx[TY][WC];           // cells rows [i0,i0+TY), cols [j0-1, j0+TX+1)
    __shared__ T s_syy[WR][TX];           // cells rows [i0-1,i0+TY+1), cols [j0, j0+TX)
    __shared__ T s_sxy[TY + 1][TX + 1];   // vertices rows [i0, i0+TY], cols [j0, j0+TX]
    __shared__ T s_detaH[TAN ? WR : 1][TAN ? WC : 1];

    const int ny = g.ny, nx = g.nx;
    const int b = blockIdx.z;
    u += b * g.nu(); v += b * g.nv(); H += b * g.nc();
    a_u += b * g.nu(); a_v += b * g.nv(); a_H += b * g.nc();
    bed += b * g.nc(); B += b * g.nc(); beta += b * g.nc(); mask += b * g.nc(); gamma += b * g.nc();
    o_u += b * g.nu(); o_v += b * g.nv(); o_H += b * g.nc();
    const TileIdx t = tile_idx<TY>();
    const T dxi = p.dxi;

    // phase 1: eta (and its tangent) on the window
    for (int k = t.tid; k < WR * WC; k += NTHR) {
        int r = k / WC, c = k - r * WC;
        int i = t.i0 - 1 + r, j = t.j0 - 1 + c;
        int ic = clampi(i, 0, ny - 1), jc = clampi(j, 0, nx - 1);
        EtaIn<T> ein = eta_inputs(u, v, ic, jc, ny, nx);
        T Bc = ldc(B, ic, jc, ny, nx);
        EtaOut<T> e = cell_eta(ein, Bc, ic, jc, ny, nx, p);
        T Hc = ldc(H, ic, jc, ny, nx);
        s_eta[r][c] = e.eta;
        s_etaH[r][c] = e.eta * Hc;
        if constexpr (TAN) {
            EtaIn<T> din = eta_inputs(a_u, a_v, ic, jc, ny, nx);
            T deta = cell_eta_tangent(e, din, Bc, ic, jc, ny, nx, p);
            s_detaH[r][c] = deta * Hc + e.eta * ldc(a_H, ic, jc, ny, nx);
        }
    }
    __syncthreads();

    // phase 2: normal stresses on cells, shear stresses on vertices
    // (value for the residual, tangent for the JVP)
    for (int k = t.tid; k < TY * WC; k += NTHR) {  // sxx
        int r = k / WC, c = k - r * WC;
        int i = t.i0 + r, j = t.j0 - 1 + c;
        T ul = ldu(u, i, j, ny, nx), ur = ldu(u, i, j + 1, ny, nx);
        T vt = ldv(v, i, j, ny, nx), vb = ldv(v, i + 1, j, ny, nx);
        NormalStress<T> s = normal_stress<T, true>(ul, ur, vt, vb, s_etaH[r + 1][c], dxi, j >= 0 && j < nx);
        if constexpr (TAN) {
            s_sxx[r][c] = s.d_ul * ldu(a_u, i, j, ny, nx) + s.d_ur * ldu(a_u, i, j + 1, ny, nx) +
                          s.d_vt * ldv(a_v, i, j, ny, nx) + s.d_vb * ldv(a_v, i + 1, j, ny, nx) +
                          s.d_etaH * s_detaH[r + 1][c];
        } else {
            s_sxx[r][c] = s.res;
        }
    }
    for (int k = t.tid; k < WR * TX; k += NTHR) {  // syy
        int r = k / TX, c = k - r * TX;
        int i = t.i0 - 1 + r, j = t.j0 + c;
        T ul = ldu(u, i, j, ny, nx), ur = ldu(u, i, j + 1, ny, nx);
        T vt = ldv(v, i, j, ny, nx), vb = ldv(v, i + 1, j, ny, nx);
        NormalStress<T> s = normal_stress<T, false>(ul, ur, vt, vb, s_etaH[r][c + 1], dxi, i >= 0 && i < ny);
        if constexpr (TAN) {
            s_syy[r][c] = s.d_ul * ldu(a_u, i, j, ny, nx) + s.d_ur * ldu(a_u, i, j + 1, ny, nx) +
                          s.d_vt * ldv(a_v, i, j, ny, nx) + s.d_vb * ldv(a_v, i + 1, j, ny, nx) +
                          s.d_etaH * s_detaH[r][c + 1];
        } else {
            s_syy[r][c] = s.res;
        }
    }
    for (int k = t.tid; k < (TY + 1) * (TX + 1); k += NTHR) {  // sxy on vertex (i,j)
        int r = k / (TX + 1), c = k - r * (TX + 1);
        int i = t.i0 + r, j = t.j0 + c;
        // cells around vertex (i,j): (i-1,j-1) (i-1,j) (i,j-1) (i,j) -> window (r,c) (r,c+1) (r+1,c) (r+1,c+1)
        T etaH = T(0.25) * (s_etaH[r][c] + s_etaH[r][c + 1] + s_etaH[r + 1][c] + s_etaH[r + 1][c + 1]);
        T ut = ldu(u, i - 1, j, ny, nx), ub = ldu(u, i, j, ny, nx);
        T vl = ldv(v, i, j - 1, ny, nx), vr = ldv(v, i, j, ny, nx);
        bool valid = i > 0 && i < ny && j > 0 && j < nx;
        ShearStress<T> s = shear_stress(ut, ub, vl, vr, etaH, dxi, valid);
        if constexpr (TAN) {
            T detaH = T(0.25) * (s_detaH[r][c] + s_detaH[r][c + 1] + s_detaH[r + 1][c] + s_detaH[r + 1][c + 1]);
            s_sxy[r][c] = s.d_ut * ldu(a_u, i - 1, j, ny, nx) + s.d_ub * ldu(a_u, i, j, ny, nx) +
                          s.d_vl * ldv(a_v, i, j - 1, ny, nx) + s.d_vr * ldv(a_v, i, j, ny, nx) +
                          s.d_etaH * detaH;
        } else {
            s_sxy[r][c] = s.res;
        }
    }
    __syncthreads();

    // phase 3: owned outputs
#pragma unroll
    for (int k = 0; k < RPT; k++) {
        const int r = t.ty + k * (NTHR / TX);
        const int c = t.tx;
        const int i = t.i0 + r, j = t.j0 + c;
        if (i >= ny || j >= nx) continue;
        const T Hc = H[int64_t(i) * nx + j];
        const T Hl = ldc(H, i, j - 1, ny, nx), Hr = ldc(H, i, j + 1, ny, nx);
        const T Ht = ldc(H, i - 1, j, ny, nx), Hb = ldc(H, i + 1, j, ny, nx);
        const T bc = bed[int64_t(i) * nx + j];
        const T bl = ldc(bed, i, j - 1, ny, nx), bt = ldc(bed, i - 1, j, ny, nx);
        const T betac = beta[int64_t(i) * nx + j];
        const T betal = ldc(beta, i, j - 1, ny, nx), betat = ldc(beta, i - 1, j, ny, nx);
        const T ul = u[int64_t(i) * (nx + 1) + j], ur = u[int64_t(i) * (nx + 1) + j + 1];
        const T vt = v[int64_t(i) * nx + j], vb = v[int64_t(i + 1) * nx + j];
        T dHc = 0, dHl = 0, dHt = 0, dHr = 0, dHb = 0, dul = 0, dur = 0, dvt = 0, dvb = 0;
        if constexpr (TAN) {
            dHc = a_H[int64_t(i) * nx + j];
            dHl = ldc(a_H, i, j - 1, ny, nx); dHr = ldc(a_H, i, j + 1, ny, nx);
            dHt = ldc(a_H, i - 1, j, ny, nx); dHb = ldc(a_H, i + 1, j, ny, nx);
            dul = a_u[int64_t(i) * (nx + 1) + j]; dur = a_u[int64_t(i) * (nx + 1) + j + 1];
            dvt = a_v[int64_t(i) * nx + j]; dvb = a_v[int64_t(i + 1) * nx + j];
        }

        // ---- mass row (residuals.cu:50-84)
        {
            const T m = mask[int64_t(i) * nx + j];
            Flux<T> ql = upwind_flux(ul, Hl, Hc, j > 0 && j < nx);
            Flux<T> qr = upwind_flux(ur, Hc, Hr, j + 1 > 0 && j + 1 < nx);
            Flux<T> qt = upwind_flux(vt, Hc, Ht, i > 0 && i < ny);         // a = bottom (this cell), b = top
            Flux<T> qb = upwind_flux(vb, Hb, Hc, i + 1 > 0 && i + 1 < ny);
            Calving<T> cv = calving(Hc, bc, p);
            if constexpr (TAN) {
                T d = dHc / p.dt - cv.d_H * dHc;
                d -= (ql.d_vel * dul + ql.d_Ha * dHl + ql.d_Hb * dHc) * dxi;
                d += (qr.d_vel * dur + qr.d_Ha * dHc + qr.d_Hb * dHr) * dxi;
                d += (qt.d_vel * dvt + qt.d_Ha * dHc + qt.d_Hb * dHt) * dxi;
                d -= (qb.d_vel * dvb + qb.d_Ha * dHb + qb.d_Hb * dHc) * dxi;
                o_H[int64_t(i) * nx + j] = (T(1) - m) * d + m * dHc;
            } else {
                T rH = Hc / p.dt - a_H[int64_t(i) * nx + j];
                rH -= cv.res;
                rH -= ql.res * dxi;
                rH += qr.res * dxi;
                rH += qt.res * dxi;
                rH -= qb.res * dxi;
                o_H[int64_t(i) * nx + j] = (T(1) - m) * rH + m * (Hc - gamma[int64_t(i) * nx + j]);
            }
        }

        // ---- u-face (i,j) and, at the right edge, (i,nx)
        for (int e = 0; e < 2; e++) {
            const int jj = j + e;
            if (e == 1 && jj != nx) break;
            const int cc = c + e;  // window column offset of cell jj is cc+1 in s_sxx
            T val = (s_sxx[r][cc + 1] - s_sxx[r][cc]) * dxi + (s_sxy[r][cc] - s_sxy[r + 1][cc]) * dxi;
            const T uf = e ? ur : ul;
            const T H1 = e ? Hc : Hl, H2 = e ? Hr : Hc;          // clamped: Hr==Hc at the edge
            const T b1 = e ? bc : bl, b2 = e ? ldc(bed, i, jj, ny, nx) : bc;
            const T be1 = e ? betac : betal, be2 = e ? ldc(beta, i, jj, ny, nx) : betac;
            BasalDrag<T> tb = basal_drag(uf, H1, H2, b1, b2, be1, be2, p);
            Driving<T> td = driving(H1, H2, b1, b2, dxi, jj > 0 && jj < nx);
            if constexpr (TAN) {
                const T duf = e ? dur : dul;
                const T dH1 = e ? dHc : dHl, dH2 = e ? dHr : dHc;
                val += tb.d_vel * duf + tb.d_H1 * dH1 + tb.d_H2 * dH2;
                val -= td.d_Hm * dH1 + td.d_Hp * dH2;
            } else {
                val += tb.res - td.res;
                val -= a_u[int64_t(i) * (nx + 1) + jj];
            }
            o_u[int64_t(i) * (nx + 1) + jj] = val;
        }
        // ---- v-face (i,j) and, at the bottom edge, (ny,j)
        for (int e = 0; e < 2; e++) {
            const int ii = i + e;
            if (e == 1 && ii != ny) break;
            const int rr = r + e;  // s_syy row of cell ii-1 is rr, of cell ii is rr+1
            T val = (s_syy[rr][c] - s_syy[rr + 1][c]) * dxi + (s_sxy[rr][c + 1] - s_sxy[rr][c]) * dxi;
            const T vf = e ? vb : vt;
            const T Htop = e ? Hc : Ht, Hbot = e ? Hb : Hc;    // clamped: Hb==Hc at the edge
            const T btop = e ? bc : bt, bbot = e ? ldc(bed, ii, j, ny, nx) : bc;
            const T betop = e ? betac : betat, bebot = e ? ldc(beta, ii, j, ny, nx) : betac;
            BasalDrag<T> tb = basal_drag(vf, Htop, Hbot, btop, bbot, betop, bebot, p);
            Driving<T> td = driving(Hbot, Htop, bbot, btop, dxi, ii > 0 && ii < ny);
            if constexpr (TAN) {
                const T dvf = e ? dvb : dvt;
                const T dtop = e ? dHc : dHt, dbot = e ? dHb : dHc;
                val += tb.d_vel * dvf + tb.d_H1 * dtop + tb.d_H2 * dbot;
                val -= td.d_Hm * dbot + td.d_Hp * dtop;
            } else {
                val += tb.res - td.res;
                val -= a_v[int64_t(ii) * nx + j];
            }
            o_v[int64_t(ii) * nx + j] = val;
        }
    }
}

// --------------------------------------------------------------------------
// residual r = F(U) - f with every input read once (glide/cuda/residuals.cu:
// 6-292).  Same tile, phases and arithmetic as stencil_kernel<T,false>, but u,
// v, H, bed and beta of the tile plus the rings the stencil needs are staged
// into shared memory first with coalesced row loads; the clamped-index rule
// is applied once while staging (a staged entry at global (i, j) holds the
// value of the clamped index), so every later read is a plain shared-memory
// read at unclamped global coordinates.
// --------------------------------------------------------------------------
constexpr int RU_R = TY + 4, RU_C = TX + 3;   // u rows [i0-2, i0+TY+2), cols [j0-1, j0+TX+2)
constexpr int RV_R = TY + 3, RV_C = TX + 4;   // v rows [i0-1, i0+TY+2), cols [j0-2, j0+TX+2)
constexpr int RC_R = TY + 2, RC_C = TX + 2;   // cells rows [i0-1, i0+TY+1), cols [j0-1, j0+TX+1)

#ifndef GLIDE_RES_MINB32
#define GLIDE_RES_MINB32 4
#endif
#ifndef GLIDE_RES_MINB64
#define GLIDE_RES_MINB64 3
#endif
template <typename T>
__global__ void __launch_bounds__(NTHR, sizeof(T) == 4 ? GLIDE_RES_MINB32 : GLIDE_RES_MINB64) residual_kernel(
    T* __restrict__ o_u, T* __restrict__ o_v, T* __restrict__ o_H,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ f_u, const T* __restrict__ f_v, const T* __restrict__ f_H,
    const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta,
    const T* __restrict__ mask, const T* __restrict__ gamma, Geo g, Phys<T> p) {
    __shared__ T s_u[RU_R][RU_C];
    __shared__ T s_v[RV_R][RV_C];
    __shared__ T s_H[RC_R][RC_C];
    __shared__ T s_bed[RC_R][RC_C];
    __shared__ T s_beta[RC_R][RC_C];
    __shared__ T s_etaH[WR][WC];
    __shared__ T s_sxx[TY][WC];           // cells rows [i0,i0+TY), cols [j0-1, j0+TX+1)
    __shared__ T s_syy[WR][TX];           // cells rows [i0-1,i0+TY+1), cols [j0, j0+TX)
    __shared__ T s_sxy[TY + 1][TX + 1];   // vertices rows [i0, i0+TY], cols [j0, j0+TX]

    const int ny = g.ny, nx = g.nx;
    const int b = blockIdx.z;
    u += b * g.nu(); v += b * g.nv(); H += b * g.nc();
    f_u += b * g.nu(); f_v += b * g.nv(); f_H += b * g.nc();
    bed += b * g.nc(); B += b * g.nc(); beta += b * g.nc(); mask += b * g.nc(); gamma += b * g.nc();
    o_u += b * g.nu(); o_v += b * g.nv(); o_H += b * g.nc();
    const TileIdx t = tile_idx<TY>();
    const T dxi = p.dxi;
    const int ur0 = t.i0 - 2, uc0 = t.j0 - 1, vr0 = t.i0 - 1, vc0 = t.j0 - 2, cr0 = t.i0 - 1, cc0 = t.j0 - 1;

    stage(&s_u[0][0], u, ny, nx + 1, ur0, uc0, RU_R, RU_C, t.tid, NTHR);
    stage(&s_v[0][0], v, ny + 1, nx, vr0, vc0, RV_R, RV_C, t.tid, NTHR);
    stage(&s_H[0][0], H, ny, nx, cr0, cc0, RC_R, RC_C, t.tid, NTHR);
    stage(&s_bed[0][0], bed, ny, nx, cr0, cc0, RC_R, RC_C, t.tid, NTHR);
    stage(&s_beta[0][0], beta, ny, nx, cr0, cc0, RC_R, RC_C, t.tid, NTHR);
    __syncthreads();
    auto U = [&](int i, int j) -> T { return s_u[i - ur0][j - uc0]; };
    auto V = [&](int i, int j) -> T { return s_v[i - vr0][j - vc0]; };

    // phase 1: eta*H on the window (cells clamped into the domain)
    for (int k = t.tid; k < WR * WC; k += NTHR) {
        int r = k / WC, c = k - r * WC;
        int ic = clampi(t.i0 - 1 + r, 0, ny - 1), jc = clampi(t.j0 - 1 + c, 0, nx - 1);
        EtaIn<T> a;
        a.ul = U(ic, jc);          a.ur = U(ic, jc + 1);
        a.vt = V(ic, jc);          a.vb = V(ic + 1, jc);
        a.u_tl = U(ic - 1, jc);    a.u_tr = U(ic - 1, jc + 1);
        a.u_bl = U(ic + 1, jc);    a.u_br = U(ic + 1, jc + 1);
        a.v_lt = V(ic, jc - 1);    a.v_rt = V(ic, jc + 1);
        a.v_lb = V(ic + 1, jc - 1); a.v_rb = V(ic + 1, jc + 1);
        EtaOut<T> e = cell_eta(a, __ldg(B + int64_t(ic) * nx + jc), ic, jc, ny, nx, p);
        s_etaH[r][c] = e.eta * s_H[ic - cr0][jc - cc0];
    }
    __syncthreads();

    // phase 2: normal stresses on cells, shear stresses on vertices
    for (int k = t.tid; k < TY * WC; k += NTHR) {
        int r = k / WC, c = k - r * WC;
        int i = t.i0 + r, j = t.j0 - 1 + c;
        s_sxx[r][c] = normal_stress<T, true>(U(i, j), U(i, j + 1), V(i, j), V(i + 1, j), s_etaH[r + 1][c], dxi,
                                             j >= 0 && j < nx).res;
    }
    for (int k = t.tid; k < WR * TX; k += NTHR) {
        int r = k / TX, c = k - r * TX;
        int i = t.i0 - 1 + r, j = t.j0 + c;
        s_syy[r][c] = normal_stress<T, false>(U(i, j), U(i, j + 1), V(i, j), V(i + 1, j), s_etaH[r][c + 1], dxi,
                                              i >= 0 && i < ny).res;
    }
    for (int k = t.tid; k < (TY + 1) * (TX + 1); k += NTHR) {
        int r = k / (TX + 1), c = k - r * (TX + 1);
        int i = t.i0 + r, j = t.j0 + c;
        T etaH = T(0.25) * (s_etaH[r][c] + s_etaH[r][c + 1] + s_etaH[r + 1][c] + s_etaH[r + 1][c + 1]);
        s_sxy[r][c] = shear_stress(U(i - 1, j), U(i, j), V(i, j - 1), V(i, j), etaH, dxi,
                                   i > 0 && i < ny && j > 0 && j < nx).res;
    }
    __syncthreads();

    // phase 3: owned outputs
#pragma unroll
    for (int k = 0; k < RPT; k++) {
        const int r = t.ty + k * (NTHR / TX);
        const int c = t.tx;
        const int i = t.i0 + r, j = t.j0 + c;
        if (i >= ny || j >= nx) continue;
        const int sr = r + 1, sc = c + 1;  // this cell in the staged cell windows
        const T Hc = s_H[sr][sc], Hl = s_H[sr][sc - 1], Hr = s_H[sr][sc + 1];
        const T Ht = s_H[sr - 1][sc], Hb = s_H[sr + 1][sc];
        const T bc = s_bed[sr][sc], bl = s_bed[sr][sc - 1], bt = s_bed[sr - 1][sc];
        const T betac = s_beta[sr][sc], betal = s_beta[sr][sc - 1], betat = s_beta[sr - 1][sc];
        const T ul = U(i, j), ur = U(i, j + 1), vt = V(i, j), vb = V(i + 1, j);
        const int64_t ic = int64_t(i) * nx + j;

        // ---- mass row (residuals.cu:50-84)
        {
            const T m = mask[ic];
            Flux<T> ql = upwind_flux(ul, Hl, Hc, j > 0 && j < nx);
            Flux<T> qr = upwind_flux(ur, Hc, Hr, j + 1 > 0 && j + 1 < nx);
            Flux<T> qt = upwind_flux(vt, Hc, Ht, i > 0 && i < ny);
            Flux<T> qb = upwind_flux(vb, Hb, Hc, i + 1 > 0 && i + 1 < ny);
            Calving<T> cv = calving(Hc, bc, p);
            T rH = Hc / p.dt - f_H[ic];
            rH -= cv.res;
            rH -= ql.res * dxi;
            rH += qr.res * dxi;
            rH += qt.res * dxi;
            rH -= qb.res * dxi;
            o_H[ic] = (T(1) - m) * rH + m * (Hc - gamma[ic]);
        }
        // ---- u-face (i,j) and, at the right edge, (i,nx)
        for (int e = 0; e < 2; e++) {
            const int jj = j + e;
            if (e == 1 && jj != nx) break;
            const int cc = c + e;
            T val = (s_sxx[r][cc + 1] - s_sxx[r][cc]) * dxi + (s_sxy[r][cc] - s_sxy[r + 1][cc]) * dxi;
            const T uf = e ? ur : ul;
            const T H1 = e ? Hc : Hl, H2 = e ? Hr : Hc;
            const T b1 = e ? bc : bl, b2 = e ? s_bed[sr][sc + 1] : bc;
            const T be1 = e ? betac : betal, be2 = e ? s_beta[sr][sc + 1] : betac;
            BasalDrag<T> tb = basal_drag(uf, H1, H2, b1, b2, be1, be2, p);
            Driving<T> td = driving(H1, H2, b1, b2, dxi, jj > 0 && jj < nx);
            val += tb.res - td.res;
            val -= f_u[int64_t(i) * (nx + 1) + jj];
            o_u[int64_t(i) * (nx + 1) + jj] = val;
        }
        // ---- v-face (i,j) and, at the bottom edge, (ny,j)
        for (int e = 0; e < 2; e++) {
            const int ii = i + e;
            if (e == 1 && ii != ny) break;
            const int rr = r + e;
            T val = (s_syy[rr][c] - s_syy[rr + 1][c]) * dxi + (s_sxy[rr][c + 1] - s_sxy[rr][c]) * dxi;
            const T vf = e ? vb : vt;
            const T Htop = e ? Hc : Ht, Hbot = e ? Hb : Hc;
            const T btop = e ? bc : bt, bbot = e ? s_bed[sr + 1][sc] : bc;
            const T betop = e ? betac : betat, bebot = e ? s_beta[sr + 1][sc] : betac;
            BasalDrag<T> tb = basal_drag(vf, Htop, Hbot, btop, bbot, betop, bebot, p);
            Driving<T> td = driving(Hbot, Htop, bbot, btop, dxi, ii > 0 && ii < ny);
            val += tb.res - td.res;
            val -= f_v[int64_t(ii) * nx + j];
            o_v[int64_t(ii) * nx + j] = val;
        }
    }
}

constexpr int VTY = 8;                   // VJP tile rows (keeps FP64 shared memory < 48 KB)
constexpr int VRPT = VTY / (NTHR / TX);  // rows per thread = 1
constexpr int VWR = VTY + 2;

// --------------------------------------------------------------------------
// VJP lambda^T J in gather form (glide/cuda/residuals.cu:586-1023)
//
// The velocity-velocity block is applied as the forward tangent with lambda
// as the direction (the viscous block is symmetric, residuals.cu:709); the
// H-row and velocity->H blocks are explicit transposes gathered per output.
// exact_boundary=0 drops the contributions the reference drops at clamped
// boundary reads (only non-zero with gl_derivatives), 1 keeps them.
// --------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NTHR) vjp_kernel(
    T* __restrict__ o_u, T* __restrict__ o_v, T* __restrict__ o_H,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ lu, const T* __restrict__ lv, const T* __restrict__ lH,
    const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta,
    const T* __restrict__ mask, const T* __restrict__ f_u, const T* __restrict__ f_v, const T* __restrict__ f_H,
    int residual_form, int exact_boundary, Geo g, Phys<T> p) {
    __shared__ T s_eta[VWR][WC];
    __shared__ T s_etaH[VWR][WC];
    __shared__ T s_detaH[VWR][WC];      // d(eta)(lambda) * H
    __shared__ T s_dsxx[VTY][WC];
    __shared__ T s_dsyy[VWR][TX];
    __shared__ T s_dsxy[VTY + 1][TX + 1];
    __shared__ T s_W[VTY + 1][TX + 1];  // vertex weight for the H rows of the shear terms
    __shared__ T s_CuL[VTY][TX + 1], s_CuR[VTY][TX + 1];
    __shared__ T s_CvT[VTY + 1][TX], s_CvB[VTY + 1][TX];

    const int ny = g.ny, nx = g.nx;
    const int b = blockIdx.z;
    u += b * g.nu(); v += b * g.nv(); H += b * g.nc();
    lu += b * g.nu(); lv += b * g.nv(); lH += b * g.nc();
    bed += b * g.nc(); B += b * g.nc(); beta += b * g.nc(); mask += b * g.nc();
    o_u += b * g.nu(); o_v += b * g.nv(); o_H += b * g.nc();
    if (residual_form) { f_u += b * g.nu(); f_v += b * g.nv(); f_H += b * g.nc(); }
    const TileIdx t = tile_idx<VTY>();
    const T dxi = p.dxi;
    auto lam_t = [&](int i, int j) -> T {  // masked lambda_H (residuals.cu:646)
        return ldc(lH, i, j, ny, nx) * (T(1) - ldc(mask, i, j, ny, nx));
    };

    for (int k = t.tid; k < VWR * WC; k += NTHR) {
        int r = k / WC, c = k - r * WC;
        int ic = clampi(t.i0 - 1 + r, 0, ny - 1), jc = clampi(t.j0 - 1 + c, 0, nx - 1);
        EtaIn<T> ein = eta_inputs(u, v, ic, jc, ny, nx);
        T Bc = ldc(B, ic, jc, ny, nx);
        EtaOut<T> e = cell_eta(ein, Bc, ic, jc, ny, nx, p);
        EtaIn<T> din = eta_inputs(lu, lv, ic, jc, ny, nx);
        T deta = cell_eta_tangent(e, din, Bc, ic, jc, ny, nx, p);
        T Hc = ldc(H, ic, jc, ny, nx);
        s_eta[r][c] = e.eta;
        s_etaH[r][c] = e.eta * Hc;
        s_detaH[r][c] = deta * Hc;
    }
    __syncthreads();

    for (int k = t.tid; k < VTY * WC; k += NTHR) {
        int r = k / WC, c = k - r * WC;
        int i = t.i0 + r, j = t.j0 - 1 + c;
        NormalStress<T> s = normal_stress<T, true>(ldu(u, i, j, ny, nx), ldu(u, i, j + 1, ny, nx),
                                                   ldv(v, i, j, ny, nx), ldv(v, i + 1, j, ny, nx),
                                                   s_etaH[r + 1][c], dxi, j >= 0 && j < nx);
        s_dsxx[r][c] = s.d_ul * ldu(lu, i, j, ny, nx) + s.d_ur * ldu(lu, i, j + 1, ny, nx) +
                       s.d_vt * ldv(lv, i, j, ny, nx) + s.d_vb * ldv(lv, i + 1, j, ny, nx) +
                       s.d_etaH * s_detaH[r + 1][c];
    }
    for (int k = t.tid; k < VWR * TX; k += NTHR) {
        int r = k / TX, c = k - r * TX;
        int i = t.i0 - 1 + r, j = t.j0 + c;
        NormalStress<T> s = normal_stress<T, false>(ldu(u, i, j, ny, nx), ldu(u, i, j + 1, ny, nx),
                                                    ldv(v, i, j, ny, nx), ldv(v, i + 1, j, ny, nx),
                                                    s_etaH[r][c + 1], dxi, i >= 0 && i < ny);
        s_dsyy[r][c] = s.d_ul * ldu(lu, i, j, ny, nx) + s.d_ur * ldu(lu, i, j + 1, ny, nx) +
                       s.d_vt * ldv(lv, i, j, ny, nx) + s.d_vb * ldv(lv, i + 1, j, ny, nx) +
                       s.d_etaH * s_detaH[r][c + 1];
    }
    for (int k = t.tid; k < (VTY + 1) * (TX + 1); k += NTHR) {
        int r = k / (TX + 1), c = k - r * (TX + 1);
        int i = t.i0 + r, j = t.j0 + c;
        T etaH = T(0.25) * (s_etaH[r][c] + s_etaH[r][c + 1] + s_etaH[r + 1][c] + s_etaH[r + 1][c + 1]);
        T detaH = T(0.25) * (s_detaH[r][c] + s_detaH[r][c + 1] + s_detaH[r + 1][c] + s_detaH[r + 1][c + 1]);
        bool valid = i > 0 && i < ny && j > 0 && j < nx;
        ShearStress<T> s = shear_stress(ldu(u, i - 1, j, ny, nx), ldu(u, i, j, ny, nx), ldv(v, i, j - 1, ny, nx),
                                        ldv(v, i, j, ny, nx), etaH, dxi, valid);
        s_dsxy[r][c] = s.d_ut * ldu(lu, i - 1, j, ny, nx) + s.d_ub * ldu(lu, i, j, ny, nx) +
                       s.d_vl * ldv(lv, i, j - 1, ny, nx) + s.d_vr * ldv(lv, i, j, ny, nx) + s.d_etaH * detaH;
        // the vertex stress enters u(i,j) [+], u(i-1,j) [-], v(i,j) [-], v(i,j-1) [+]
        T w = valid ? (ldu(lu, i, j, ny, nx) - ldu(lu, i - 1, j, ny, nx) - ldv(lv, i, j, ny, nx) +
                       ldv(lv, i, j - 1, ny, nx)) * dxi
                    : T(0);
        s_W[r][c] = w * s.d_etaH * T(0.25);
    }
    // face contributions to the H rows of their two cells
    for (int k = t.tid; k < VTY * (TX + 1); k += NTHR) {  // u-faces (i,j), j in [j0, j0+TX]
        int r = k / (TX + 1), c = k - r * (TX + 1);
        int i = t.i0 + r, j = t.j0 + c;
        T CL = 0, CR = 0;
        if (i < ny && j <= nx) {
            T uf = ldu(u, i, j, ny, nx), lam = ldu(lu, i, j, ny, nx);
            T H1 = ldc(H, i, j - 1, ny, nx), H2 = ldc(H, i, j, ny, nx);
            T b1 = ldc(bed, i, j - 1, ny, nx), b2 = ldc(bed, i, j, ny, nx);
            Flux<T> q = upwind_flux(uf, H1, H2, j > 0 && j < nx);
            T a = (lam_t(i, j - 1) - lam_t(i, j)) * dxi;
            BasalDrag<T> tb = basal_drag(uf, H1, H2, b1, b2, ldc(beta, i, j - 1, ny, nx), ldc(beta, i, j, ny, nx), p);
            Driving<T> td = driving(H1, H2, b1, b2, dxi, j > 0 && j < nx);
            CL = a * q.d_Ha + lam * (tb.d_H1 - td.d_Hm);
            CR = a * q.d_Hb + lam * (tb.d_H2 - td.d_Hp);
        }
        s_CuL[r][c] = CL;
        s_CuR[r][c] = CR;
    }
    for (int k = t.tid; k < (VTY + 1) * TX; k += NTHR) {  // v-faces (i,j), i in [i0, i0+VTY]
        int r = k / TX, c = k - r * TX;
        int i = t.i0 + r, j = t.j0 + c;
        T CT = 0, CB = 0;
        if (i <= ny && j < nx) {
            T vf = ldv(v, i, j, ny, nx), lam = ldv(lv, i, j, ny, nx);
            T Htop = ldc(H, i - 1, j, ny, nx), Hbot = ldc(H, i, j, ny, nx);
            T btop = ldc(bed, i - 1, j, ny, nx), bbot = ldc(bed, i, j, ny, nx);
            Flux<T> q = upwind_flux(vf, Hbot, Htop, i > 0 && i < ny);
            T a = (lam_t(i, j) - lam_t(i - 1, j)) * dxi;
            BasalDrag<T> tb = basal_drag(vf, Htop, Hbot, btop, bbot, ldc(beta, i - 1, j, ny, nx),
                                         ldc(beta, i, j, ny, nx), p);
            Driving<T> td = driving(Hbot, Htop, bbot, btop, dxi, i > 0 && i < ny);
            CT = a * q.d_Hb + lam * (tb.d_H1 - td.d_Hp);
            CB = a * q.d_Ha + lam * (tb.d_H2 - td.d_Hm);
        }
        s_CvT[r][c] = CT;
        s_CvB[r][c] = CB;
    }
    __syncthreads();

#pragma unroll
    for (int k = 0; k < VRPT; k++) {
        const int r = t.ty + k * (NTHR / TX);
        const int c = t.tx;
        const int i = t.i0 + r, j = t.j0 + c;
        if (i >= ny || j >= nx) continue;
        const int64_t ic = int64_t(i) * nx + j;
        // ---- H row
        {
            const T m = mask[ic];
            const T lam = lH[ic];
            const T lamt = lam * (T(1) - m);
            const T Hc = H[ic];
            Calving<T> cv = calving(Hc, bed[ic], p);
            T acc = lamt / p.dt - lamt * cv.d_H;
            acc += s_CuR[r][c] + s_CuL[r][c + 1] + s_CvB[r][c] + s_CvT[r + 1][c];
            if (exact_boundary) {
                if (j == 0) acc += s_CuL[r][c];            // face 0 read H(i,-1) -> H(i,0)
                if (j == nx - 1) acc += s_CuR[r][c + 1];   // face nx read H(i,nx) -> H(i,nx-1)
                if (i == 0) acc += s_CvT[r][c];
                if (i == ny - 1) acc += s_CvB[r + 1][c];
            }
            const T eta = s_eta[r + 1][c + 1], etaH = s_etaH[r + 1][c + 1];
            const T ul = u[int64_t(i) * (nx + 1) + j], ur = u[int64_t(i) * (nx + 1) + j + 1];
            const T vt = v[ic], vb = v[int64_t(i + 1) * nx + j];
            NormalStress<T> sx = normal_stress<T, true>(ul, ur, vt, vb, etaH, dxi, true);
            NormalStress<T> sy = normal_stress<T, false>(ul, ur, vt, vb, etaH, dxi, true);
            const T lul = lu[int64_t(i) * (nx + 1) + j], lur = lu[int64_t(i) * (nx + 1) + j + 1];
            const T lvt = lv[ic], lvb = lv[int64_t(i + 1) * nx + j];
            acc += (lul - lur) * sx.d_etaH * eta * dxi;
            acc += (lvb - lvt) * sy.d_etaH * eta * dxi;
            acc += eta * (s_W[r][c] + s_W[r][c + 1] + s_W[r + 1][c] + s_W[r + 1][c + 1]);
            acc += lam * m;
            o_H[ic] = residual_form ? f_H[ic] - acc : acc;
        }
        // ---- u-faces
        for (int e = 0; e < 2; e++) {
            const int jj = j + e;
            if (e == 1 && jj != nx) break;
            const int cc = c + e;
            T val = (s_dsxx[r][cc + 1] - s_dsxx[r][cc]) * dxi + (s_dsxy[r][cc] - s_dsxy[r + 1][cc]) * dxi;
            const T uf = ldu(u, i, jj, ny, nx), lam = ldu(lu, i, jj, ny, nx);
            const T H1 = ldc(H, i, jj - 1, ny, nx), H2 = ldc(H, i, jj, ny, nx);
            BasalDrag<T> tb = basal_drag(uf, H1, H2, ldc(bed, i, jj - 1, ny, nx), ldc(bed, i, jj, ny, nx),
                                         ldc(beta, i, jj - 1, ny, nx), ldc(beta, i, jj, ny, nx), p);
            Flux<T> q = upwind_flux(uf, H1, H2, jj > 0 && jj < nx);
            val += lam * tb.d_vel + (lam_t(i, jj - 1) - lam_t(i, jj)) * dxi * q.d_vel;
            const int64_t iu = int64_t(i) * (nx + 1) + jj;
            o_u[iu] = residual_form ? f_u[iu] - val : val;
        }
        // ---- v-faces
        for (int e = 0; e < 2; e++) {
            const int ii = i + e;
            if (e == 1 && ii != ny) break;
            const int rr = r + e;
            T val = (s_dsyy[rr][c] - s_dsyy[rr + 1][c]) * dxi + (s_dsxy[rr][c + 1] - s_dsxy[rr][c]) * dxi;
            const T vf = ldv(v, ii, j, ny, nx), lam = ldv(lv, ii, j, ny, nx);
            const T Htop = ldc(H, ii - 1, j, ny, nx), Hbot = ldc(H, ii, j, ny, nx);
            BasalDrag<T> tb = basal_drag(vf, Htop, Hbot, ldc(bed, ii - 1, j, ny, nx), ldc(bed, ii, j, ny, nx),
                                         ldc(beta, ii - 1, j, ny, nx), ldc(beta, ii, j, ny, nx), p);
            Flux<T> q = upwind_flux(vf, Hbot, Htop, ii > 0 && ii < ny);
            val += lam * tb.d_vel + (lam_t(ii, j) - lam_t(ii - 1, j)) * dxi * q.d_vel;
            const int64_t iv = int64_t(ii) * nx + j;
            o_v[iv] = residual_form ? f_v[iv] - val : val;
        }
    }
}

// --------------------------------------------------------------------------
// grad_beta[c] = sum_faces lambda_face d tau_b / d beta_c  (glide/cuda/grad.cu)
// exact_boundary=0 reproduces the reference's j>0 / j<nx-1 (and i) guards
// (grad.cu:52-53, :70-71); 1 sends every term to the cell it was read from.
// --------------------------------------------------------------------------
template <typename T>
__global__ void grad_beta_kernel(T* __restrict__ grad, const T* __restrict__ u, const T* __restrict__ v,
                                 const T* __restrict__ H, const T* __restrict__ lu, const T* __restrict__ lv,
                                 const T* __restrict__ bed, const T* __restrict__ beta, int exact_boundary,
                                 Geo g, Phys<T> p) {
    const int ny = g.ny, nx = g.nx;
    const int b = blockIdx.z;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= ny || j >= nx) return;
    u += b * g.nu(); v += b * g.nv(); H += b * g.nc(); lu += b * g.nu(); lv += b * g.nv();
    bed += b * g.nc(); beta += b * g.nc(); grad += b * g.nc();
    T acc = 0;
    auto uface = [&](int jj) {
        return basal_drag(ldu(u, i, jj, ny, nx), ldc(H, i, jj - 1, ny, nx), ldc(H, i, jj, ny, nx),
                          ldc(bed, i, jj - 1, ny, nx), ldc(bed, i, jj, ny, nx), ldc(beta, i, jj - 1, ny, nx),
                          ldc(beta, i, jj, ny, nx), p);
    };
    auto vface = [&](int ii) {
        return basal_drag(ldv(v, ii, j, ny, nx), ldc(H, ii - 1, j, ny, nx), ldc(H, ii, j, ny, nx),
                          ldc(bed, ii - 1, j, ny, nx), ldc(bed, ii, j, ny, nx), ldc(beta, ii - 1, j, ny, nx),
                          ldc(beta, ii, j, ny, nx), p);
    };
    // right face (i,j+1): this cell is its left cell (added when j+1 > 0: always)
    acc += ldu(lu, i, j + 1, ny, nx) * uface(j + 1).d_beta1;
    // left face (i,j): this cell is its right cell (reference adds it only for j < nx-1)
    if (exact_boundary || j < nx - 1) acc += ldu(lu, i, j, ny, nx) * uface(j).d_beta2;
    if (exact_boundary && j == 0) acc += ldu(lu, i, 0, ny, nx) * uface(0).d_beta1;
    if (exact_boundary && j == nx - 1) acc += ldu(lu, i, nx, ny, nx) * uface(nx).d_beta2;
    acc += ldv(lv, i + 1, j, ny, nx) * vface(i + 1).d_beta1;
    if (exact_boundary || i < ny - 1) acc += ldv(lv, i, j, ny, nx) * vface(i).d_beta2;
    if (exact_boundary && i == 0) acc += ldv(lv, 0, j, ny, nx) * vface(0).d_beta1;
    if (exact_boundary && i == ny - 1) acc += ldv(lv, ny, j, ny, nx) * vface(ny).d_beta2;
    grad[int64_t(i) * nx + j] = acc;
}

// --------------------------------------------------------------------------
// launchers
// --------------------------------------------------------------------------
static inline dim3 tile_grid(const Geo& g, int ty = TY) { return dim3((g.nx + TX - 1) / TX, (g.ny + ty - 1) / ty, g.nb); }

template <typename T>
int launch_residual(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, void* r_u, void* r_v,
                    void* r_H, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    glide::count_launch(), residual_kernel<T><<<tile_grid(g), NTHR, 0, s>>>(
        (T*)r_u, (T*)r_v, (T*)r_H, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)f_u, (const T*)f_v,
        (const T*)f_H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->mask,
        (const T*)a->gamma, g, p);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_jvp(const GlideLevelArgs* a, const void* d_u, const void* d_v, const void* d_H, void* j_u, void* j_v,
               void* j_H, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    glide::count_launch(), stencil_kernel<T, true><<<tile_grid(g), NTHR, 0, s>>>(
        (T*)j_u, (T*)j_v, (T*)j_H, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)d_u, (const T*)d_v,
        (const T*)d_H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->mask,
        (const T*)a->gamma, g, p);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_vjp(const GlideLevelArgs* a, const void* l_u, const void* l_v, const void* l_H, const void* f_u,
               const void* f_v, const void* f_H, void* o_u, void* o_v, void* o_H, int exact_boundary,
               cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    int rf = f_u != nullptr;
    glide::count_launch(), vjp_kernel<T><<<tile_grid(g, VTY), NTHR, 0, s>>>(
        (T*)o_u, (T*)o_v, (T*)o_H, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)l_u, (const T*)l_v,
        (const T*)l_H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->mask, (const T*)f_u,
        (const T*)f_v, (const T*)f_H, rf, exact_boundary, g, p);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_grad_beta(const GlideLevelArgs* a, const void* l_u, const void* l_v, void* grad, int exact_boundary,
                     cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    dim3 blk(32, 8);
    dim3 grd((g.nx + 31) / 32, (g.ny + 7) / 8, g.nb);
    glide::count_launch(), grad_beta_kernel<T><<<grd, blk, 0, s>>>((T*)grad, (const T*)a->u, (const T*)a->v, (const T*)a->H,
                                            (const T*)l_u, (const T*)l_v, (const T*)a->bed, (const T*)a->beta,
                                            exact_boundary, g, p);
    return (int)cudaGetLastError();
}

template int launch_residual<float>(const GlideLevelArgs*, const void*, const void*, const void*, void*, void*, void*,
                                    cudaStream_t);
template int launch_residual<double>(const GlideLevelArgs*, const void*, const void*, const void*, void*, void*,
                                     void*, cudaStream_t);
template int launch_jvp<float>(const GlideLevelArgs*, const void*, const void*, const void*, void*, void*, void*,
                               cudaStream_t);
template int launch_jvp<double>(const GlideLevelArgs*, const void*, const void*, const void*, void*, void*, void*,
                                cudaStream_t);
template int launch_vjp<float>(const GlideLevelArgs*, const void*, const void*, const void*, const void*, const void*,
                               const void*, void*, void*, void*, int, cudaStream_t);
template int launch_vjp<double>(const GlideLevelArgs*, const void*, const void*, const void*, const void*,
                                const void*, const void*, void*, void*, void*, int, cudaStream_t);
template int launch_grad_beta<float>(const GlideLevelArgs*, const void*, const void*, void*, int, cudaStream_t);
template int launch_grad_beta<double>(const GlideLevelArgs*, const void*, const void*, void*, int, cudaStream_t);

}  // namespace glide
