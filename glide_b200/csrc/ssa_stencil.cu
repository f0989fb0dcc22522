// Residual, JVP, VJP and basal-friction gradient kernels for the SSA system
// on the MAC staggered grid.
//
// Structure (B200): the residual, the JVP and the VJP stream -- a warp owns a
// strip of cell columns and marches down the rows, holding the neighbouring
// rows in registers and the neighbouring columns in its lanes (warp
// shuffles), so each input is read once per launch and no shared memory or
// barrier is needed.  Every output has exactly one writer, so results are
// deterministic (the reference scatters its VJP with float atomics,
// glide/cuda/residuals.cu:617-1021).
#include "glide_common.cuh"

namespace glide {

// --------------------------------------------------------------------------
// residual, streaming form (what launch_residual runs).  A warp owns a strip
// of SW = 30 cell columns plus one halo column on each side (lane l holds
// column j0 - 1 + l) and marches down a chunk of rows.  Everything the
// stencil needs from the rows above and below stays in registers (u, v for 3
// rows, H / grounded fraction / surface / beta for 3 cell rows, eta*H for 2,
// the previous row's syy and vertex sxy); horizontal neighbours come from
// warp shuffles.  Per row each input field is read once (coalesced), each
// output written once, and the grounding sigmoid and the surface are computed
// once per cell instead of once per face.  Loads use clamped rows and
// per-lane clamped columns, so every in-domain value equals the clamped
// accessors'; values of out-of-domain cells only enter terms their validity
// flags zero.  Same arithmetic as the reference's residual
// (glide/cuda/residuals.cu:6-579).
// --------------------------------------------------------------------------
constexpr int SW = 30;

template <typename T>
__device__ __forceinline__ T driving_s(T Hm, T Hp, T Sm, T Sp, T dxi, bool valid) {
    const T w = valid ? T(1) : T(0);
    const T Havg = T(0.5) * (Hm + Hp);
    const T dS = Sp - Sm;
    return Havg * dS * dxi * w;
}

#ifndef GLIDE_RS_MINB32
#define GLIDE_RS_MINB32 2
#endif
#ifndef GLIDE_RS_MINB64
#define GLIDE_RS_MINB64 2
#endif
// Ix: the element-index type of the per-field offsets (int when every field
// has fewer than 2^31 elements, which keeps the address arithmetic 32-bit).
template <typename T, typename Ix>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? GLIDE_RS_MINB32 : GLIDE_RS_MINB64) residual_stream_kernel(
    T* __restrict__ o_u, T* __restrict__ o_v, T* __restrict__ o_H,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ f_u, const T* __restrict__ f_v, const T* __restrict__ f_H,
    const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta,
    const T* __restrict__ mask, const T* __restrict__ gamma, Geo g, Phys<T> p, int n_strips, int rows, int n_warps) {
    const int ny = g.ny, nx = g.nx;
    const int wid = blockIdx.x * (256 / 32) + threadIdx.x / 32;
    if (wid >= n_warps) return;  // whole warp
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.y;
    u += b * g.nu(); v += b * g.nv(); H += b * g.nc();
    f_u += b * g.nu(); f_v += b * g.nv(); f_H += b * g.nc();
    bed += b * g.nc(); B += b * g.nc(); beta += b * g.nc(); mask += b * g.nc(); gamma += b * g.nc();
    o_u += b * g.nu(); o_v += b * g.nv(); o_H += b * g.nc();

    const int strip = wid % n_strips, chunk = wid / n_strips;
    const int i0 = chunk * rows;
    const int i1 = min(i0 + rows, ny);
    const int jc = strip * SW - 1 + lane;           // this lane's cell column
    const int jcc = clampi(jc, 0, nx - 1);          // clamped cell / v column
    const int juL = clampi(jc, 0, nx);              // this lane's left u-face
    const int juR = clampi(jc + 1, 0, nx);          // right u-face (own load on lane 31)
    const int jvL = clampi(jc - 1, 0, nx - 1), jvR = clampi(jc + 1, 0, nx - 1);
    const bool first = lane == 0, last = lane == 31;
    const bool own = lane >= 1 && lane <= SW && jc < nx;
    const unsigned FULL = 0xffffffffu;
    const T dxi = p.dxi;
    const T rr = rho_ratio<T>();
    auto U = [&](int r, int col) -> T { return __ldg(u + Ix(clampi(r, 0, ny - 1)) * (nx + 1) + col); };
    auto Vf = [&](int r, int col) -> T { return __ldg(v + Ix(clampi(r, 0, ny)) * nx + col); };
    auto Cell = [&](const T* a, int r) -> T { return __ldg(a + Ix(clampi(r, 0, ny - 1)) * nx + jcc); };

    // state at the start of iteration i: u, v rows i and i+1; cell rows i-1 and i;
    // eta*H of row i; vertex sxy of row i; syy of row i-1
    int i = i0 - 2;
    T uL0 = U(i, juL), uL1 = U(i + 1, juL);
    T uR0 = last ? U(i, juR) : T(0), uR1 = last ? U(i + 1, juR) : T(0);
    T v0 = Vf(i, jcc), v1 = Vf(i + 1, jcc);
    T vL1 = first ? Vf(i + 1, jvL) : T(0), vR1 = last ? Vf(i + 1, jvR) : T(0);
    T Hm = T(0), gm = T(0), Sm = T(0), bem = T(0);
    T Hc = T(0), gcc = T(0), Sc = T(0), bec = T(0);
    T etaH0 = T(0), sxy0 = T(0), syym = T(0);
    // inputs of iteration k: u, v of row k+2, cell fields of row k+1, the
    // right-hand side, mask and gamma of output row k.  In FP32 they are
    // loaded one iteration ahead (software prefetch: two rows of loads in
    // flight per warp); in FP64 the extra registers would spill.
    constexpr bool PREFETCH = sizeof(T) == 4;
    const int jo = jc < nx ? (jc < 0 ? 0 : jc) : nx - 1;  // output column, in range for every lane
    struct RowIn {
        T uL2, uR2, v2, vL2, vR2, H, bed, beta, B, fu, fv, fH, m, gam;
    };
    auto load_row = [&](int k) {
        RowIn r;
        r.uL2 = U(k + 2, juL);
        r.uR2 = last ? U(k + 2, juR) : T(0);
        r.v2 = Vf(k + 2, jcc);
        r.vL2 = first ? Vf(k + 2, jvL) : T(0);
        r.vR2 = last ? Vf(k + 2, jvR) : T(0);
        r.H = Cell(H, k + 1); r.bed = Cell(bed, k + 1); r.beta = Cell(beta, k + 1); r.B = Cell(B, k + 1);
        const Ix ro = clampi(k, 0, ny - 1);
        r.fu = __ldg(f_u + ro * (nx + 1) + jo);
        r.fv = __ldg(f_v + ro * nx + jo);
        r.fH = __ldg(f_H + ro * nx + jo);
        r.m = __ldg(mask + ro * nx + jo);
        r.gam = __ldg(gamma + ro * nx + jo);
        return r;
    };
    RowIn nxt;
    if constexpr (PREFETCH) nxt = load_row(i);
    for (; i < i1; ++i) {
        RowIn cur;
        if constexpr (PREFETCH) {
            cur = nxt;
            nxt = load_row(i + 1);
        } else {
            cur = load_row(i);
        }
        const T uL2 = cur.uL2, uR2 = cur.uR2, v2 = cur.v2, vL2 = cur.vL2, vR2 = cur.vR2;
        const T Hp = cur.H, bedp = cur.bed, betap = cur.beta, Bp = cur.B;
        const T fu_i = cur.fu, fv_i = cur.fv, fH_i = cur.fH, m_i = cur.m, gam_i = cur.gam;

        T uR0s = __shfl_down_sync(FULL, uL0, 1), uR1s = __shfl_down_sync(FULL, uL1, 1);
        T uR2s = __shfl_down_sync(FULL, uL2, 1);
        T vL1s = __shfl_up_sync(FULL, v1, 1), vL2s = __shfl_up_sync(FULL, v2, 1);
        T vR1s = __shfl_down_sync(FULL, v1, 1), vR2s = __shfl_down_sync(FULL, v2, 1);
        if (last) { uR0s = uR0; uR1s = uR1; uR2s = uR2; vR1s = vR1; vR2s = vR2; }
        if (first) { vL1s = vL1; vL2s = vL2; }

        // cell row i+1: grounded fraction, surface, eta*H
        const T gp = sigmoid(bedp + rr * Hp, p.sig_c);
        const T Sp = M<T>::max(bedp, -rr * Hp) + Hp;
        EtaIn<T> a;
        a.ul = uL1;   a.ur = uR1s;  a.vt = v1;    a.vb = v2;
        a.u_tl = uL0; a.u_tr = uR0s; a.u_bl = uL2; a.u_br = uR2s;
        a.v_lt = vL1s; a.v_rt = vR1s; a.v_lb = vL2s; a.v_rb = vR2s;
        const T etaHp = cell_eta(a, Bp, clampi(i + 1, 0, ny - 1), jcc, ny, nx, p).eta * Hp;

        // stresses of row i and vertex sxy of row i+1
        const T sxx = normal_stress<T, true>(uL0, uR0s, v0, v1, etaH0, dxi, jc >= 0 && jc < nx).res;
        const T syy = normal_stress<T, false>(uL0, uR0s, v0, v1, etaH0, dxi, i >= 0 && i < ny).res;
        const T etaH0L = __shfl_up_sync(FULL, etaH0, 1), etaHpL = __shfl_up_sync(FULL, etaHp, 1);
        const T sxy1 = shear_stress(uL0, uL1, vL1s, v1, T(0.25) * (etaH0L + etaH0 + etaHpL + etaHp), dxi,
                                    i + 1 > 0 && i + 1 < ny && jc > 0 && jc < nx).res;

        if (i >= i0) {  // warp-uniform
            const T sxxL = __shfl_up_sync(FULL, sxx, 1), sxxR = __shfl_down_sync(FULL, sxx, 1);
            const T sxy0R = __shfl_down_sync(FULL, sxy0, 1), sxy1R = __shfl_down_sync(FULL, sxy1, 1);
            const T HcL = __shfl_up_sync(FULL, Hc, 1), HcR = __shfl_down_sync(FULL, Hc, 1);
            const T gcL = __shfl_up_sync(FULL, gcc, 1), gcR = __shfl_down_sync(FULL, gcc, 1);
            const T ScL = __shfl_up_sync(FULL, Sc, 1);
            const T becL = __shfl_up_sync(FULL, bec, 1), becR = __shfl_down_sync(FULL, bec, 1);
            if (own) {
                const Ix ic = Ix(i) * nx + jc;
                // ---- mass row (residuals.cu:50-84)
                {
                    const T m = m_i;
                    const Flux<T> ql = upwind_flux(uL0, HcL, Hc, jc > 0 && jc < nx);
                    const Flux<T> qr = upwind_flux(uR0s, Hc, HcR, jc + 1 > 0 && jc + 1 < nx);
                    const Flux<T> qt = upwind_flux(v0, Hc, Hm, i > 0 && i < ny);
                    const Flux<T> qb = upwind_flux(v1, Hp, Hc, i + 1 > 0 && i + 1 < ny);
                    const Calving<T> cv = calving_g(Hc, gcc, p);
                    T rH = Hc / p.dt - fH_i;
                    rH -= cv.res;
                    rH -= ql.res * dxi;
                    rH += qr.res * dxi;
                    rH += qt.res * dxi;
                    rH -= qb.res * dxi;
                    o_H[ic] = (T(1) - m) * rH + m * (Hc - gam_i);
                }
                // ---- u-face (i, jc) and, at the right edge, (i, nx)
                {
                    T val = (sxx - sxxL) * dxi + (sxy0 - sxy1) * dxi;
                    val += basal_drag_g(uL0, gcL, gcc, becL, bec, p).res -
                           driving_s(HcL, Hc, ScL, Sc, dxi, jc > 0 && jc < nx);
                    val -= fu_i;
                    o_u[Ix(i) * (nx + 1) + jc] = val;
                    if (jc == nx - 1) {
                        T ve = (sxxR - sxx) * dxi + (sxy0R - sxy1R) * dxi;
                        ve += basal_drag_g(uR0s, gcc, gcR, bec, becR, p).res - T(0) * dxi;
                        ve -= f_u[Ix(i) * (nx + 1) + nx];
                        o_u[Ix(i) * (nx + 1) + nx] = ve;
                    }
                }
                // ---- v-face (i, jc) and, at the bottom edge, (ny, jc)
                {
                    T val = (syym - syy) * dxi + (sxy0R - sxy0) * dxi;
                    val += basal_drag_g(v0, gm, gcc, bem, bec, p).res -
                           driving_s(Hc, Hm, Sc, Sm, dxi, i > 0 && i < ny);
                    val -= fv_i;
                    o_v[ic] = val;
                    if (i == ny - 1) {
                        T ve = (syy - T(0)) * dxi + (sxy1R - sxy1) * dxi;
                        ve += basal_drag_g(v1, gcc, gp, bec, betap, p).res - T(0) * dxi;
                        ve -= f_v[Ix(ny) * nx + jc];
                        o_v[Ix(ny) * nx + jc] = ve;
                    }
                }
            }
        }
        // roll the window one row down
        syym = syy; sxy0 = sxy1; etaH0 = etaHp;
        Hm = Hc; gm = gcc; Sm = Sc; bem = bec;
        Hc = Hp; gcc = gp; Sc = Sp; bec = betap;
        uL0 = uL1; uL1 = uL2; uR0 = uR1; uR1 = uR2;
        v0 = v1; v1 = v2; vL1 = vL2; vR1 = vR2;
    }
}

// --------------------------------------------------------------------------
// JVP J(U) d, streaming form (what launch_jvp runs): the warp-strip march of
// residual_stream_kernel carrying the direction (d_u, d_v, d_H) beside the
// state, with the tangent of every term of the residual
// (glide/cuda/residuals.cu:299-579).  Per cell of row i+1 the
// kernel forms eta, its tangent and the tangent of eta*H once; per face the
// drag and driving partials come from the per-cell grounded fraction and the
// per-cell slope factor dS/dH = 1 + d max(bed, -rho H)/dH.  With ADD the
// output is base + J d (the linear residual of a defect correction, one pass
// instead of a JVP and a vector sum).
// --------------------------------------------------------------------------
#ifndef GLIDE_JS_MINB32
#define GLIDE_JS_MINB32 2
#endif
#ifndef GLIDE_JS_MINB64
#define GLIDE_JS_MINB64 1
#endif
template <typename T, bool ADD, typename Ix>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? GLIDE_JS_MINB32 : GLIDE_JS_MINB64) jvp_stream_kernel(
    T* __restrict__ o_u, T* __restrict__ o_v, T* __restrict__ o_H,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ d_u, const T* __restrict__ d_v, const T* __restrict__ d_H,
    const T* __restrict__ base_u, const T* __restrict__ base_v, const T* __restrict__ base_H,
    const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta,
    const T* __restrict__ mask, Geo g, Phys<T> p, int n_strips, int rows, int n_warps) {
    const int ny = g.ny, nx = g.nx;
    const int wid = blockIdx.x * (256 / 32) + threadIdx.x / 32;
    if (wid >= n_warps) return;  // whole warp
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.y;
    u += b * g.nu(); v += b * g.nv(); H += b * g.nc();
    d_u += b * g.nu(); d_v += b * g.nv(); d_H += b * g.nc();
    if constexpr (ADD) { base_u += b * g.nu(); base_v += b * g.nv(); base_H += b * g.nc(); }
    bed += b * g.nc(); B += b * g.nc(); beta += b * g.nc(); mask += b * g.nc();
    o_u += b * g.nu(); o_v += b * g.nv(); o_H += b * g.nc();

    const int strip = wid % n_strips, chunk = wid / n_strips;
    const int i0 = chunk * rows;
    const int i1 = min(i0 + rows, ny);
    const int jc = strip * SW - 1 + lane;
    const int jcc = clampi(jc, 0, nx - 1);
    const int juL = clampi(jc, 0, nx);
    const int juR = clampi(jc + 1, 0, nx);
    const int jvL = clampi(jc - 1, 0, nx - 1), jvR = clampi(jc + 1, 0, nx - 1);
    const bool first = lane == 0, last = lane == 31;
    const bool own = lane >= 1 && lane <= SW && jc < nx;
    const unsigned FULL = 0xffffffffu;
    const T dxi = p.dxi;
    const T rr = rho_ratio<T>();
    auto Uf = [&](const T* a, int r, int col) -> T {
        return __ldg(a + Ix(clampi(r, 0, ny - 1)) * (nx + 1) + col);
    };
    auto Vf = [&](const T* a, int r, int col) -> T { return __ldg(a + Ix(clampi(r, 0, ny)) * nx + col); };
    auto Cell = [&](const T* a, int r) -> T { return __ldg(a + Ix(clampi(r, 0, ny - 1)) * nx + jcc); };
    // slope factor of the surface max(bed, -rho H) + H with respect to H
    auto slope = [&](T Hx, T bx) -> T { return T(1) + (bx > -rr * Hx ? T(0) : -rr); };

    int i = i0 - 2;
    T uL0 = Uf(u, i, juL), uL1 = Uf(u, i + 1, juL);
    T uR0 = last ? Uf(u, i, juR) : T(0), uR1 = last ? Uf(u, i + 1, juR) : T(0);
    T v0 = Vf(v, i, jcc), v1 = Vf(v, i + 1, jcc);
    T vL1 = first ? Vf(v, i + 1, jvL) : T(0), vR1 = last ? Vf(v, i + 1, jvR) : T(0);
    T duL0 = Uf(d_u, i, juL), duL1 = Uf(d_u, i + 1, juL);
    T duR0 = last ? Uf(d_u, i, juR) : T(0), duR1 = last ? Uf(d_u, i + 1, juR) : T(0);
    T dv0 = Vf(d_v, i, jcc), dv1 = Vf(d_v, i + 1, jcc);
    T dvL1 = first ? Vf(d_v, i + 1, jvL) : T(0), dvR1 = last ? Vf(d_v, i + 1, jvR) : T(0);
    T Hm = T(0), gm = T(0), Sm = T(0), bem = T(0), kHm = T(0), dHm = T(0);
    T Hc = T(0), gcc = T(0), Sc = T(0), bec = T(0), kHc = T(0), dHc = T(0);
    T etaH0 = T(0), detaH0 = T(0), dsxy0 = T(0), dsyym = T(0);
    constexpr bool PREFETCH = sizeof(T) == 4;
    const int jo = jc < nx ? (jc < 0 ? 0 : jc) : nx - 1;
    struct RowIn {
        T uL2, uR2, v2, vL2, vR2, duL2, duR2, dv2, dvL2, dvR2, H, bed, beta, B, dH, m, bu, bv, bH;
    };
    auto load_row = [&](int k) {
        RowIn r;
        r.uL2 = Uf(u, k + 2, juL);
        r.uR2 = last ? Uf(u, k + 2, juR) : T(0);
        r.v2 = Vf(v, k + 2, jcc);
        r.vL2 = first ? Vf(v, k + 2, jvL) : T(0);
        r.vR2 = last ? Vf(v, k + 2, jvR) : T(0);
        r.duL2 = Uf(d_u, k + 2, juL);
        r.duR2 = last ? Uf(d_u, k + 2, juR) : T(0);
        r.dv2 = Vf(d_v, k + 2, jcc);
        r.dvL2 = first ? Vf(d_v, k + 2, jvL) : T(0);
        r.dvR2 = last ? Vf(d_v, k + 2, jvR) : T(0);
        r.H = Cell(H, k + 1); r.bed = Cell(bed, k + 1); r.beta = Cell(beta, k + 1); r.B = Cell(B, k + 1);
        r.dH = Cell(d_H, k + 1);
        const Ix ro = clampi(k, 0, ny - 1);
        r.m = __ldg(mask + ro * nx + jo);
        if constexpr (ADD) {
            r.bu = __ldg(base_u + ro * (nx + 1) + jo);
            r.bv = __ldg(base_v + ro * nx + jo);
            r.bH = __ldg(base_H + ro * nx + jo);
        } else {
            r.bu = r.bv = r.bH = T(0);
        }
        return r;
    };
    RowIn nxt;
    if constexpr (PREFETCH) nxt = load_row(i);
    for (; i < i1; ++i) {
        RowIn cur;
        if constexpr (PREFETCH) {
            cur = nxt;
            nxt = load_row(i + 1);
        } else {
            cur = load_row(i);
        }
        const T Hp = cur.H, bedp = cur.bed, betap = cur.beta, Bp = cur.B, dHp = cur.dH;

        T uR0s = __shfl_down_sync(FULL, uL0, 1), uR1s = __shfl_down_sync(FULL, uL1, 1);
        T uR2s = __shfl_down_sync(FULL, cur.uL2, 1);
        T vL1s = __shfl_up_sync(FULL, v1, 1), vL2s = __shfl_up_sync(FULL, cur.v2, 1);
        T vR1s = __shfl_down_sync(FULL, v1, 1), vR2s = __shfl_down_sync(FULL, cur.v2, 1);
        T duR0s = __shfl_down_sync(FULL, duL0, 1), duR1s = __shfl_down_sync(FULL, duL1, 1);
        T duR2s = __shfl_down_sync(FULL, cur.duL2, 1);
        T dvL1s = __shfl_up_sync(FULL, dv1, 1), dvL2s = __shfl_up_sync(FULL, cur.dv2, 1);
        T dvR1s = __shfl_down_sync(FULL, dv1, 1), dvR2s = __shfl_down_sync(FULL, cur.dv2, 1);
        if (last) {
            uR0s = uR0; uR1s = uR1; uR2s = cur.uR2; vR1s = vR1; vR2s = cur.vR2;
            duR0s = duR0; duR1s = duR1; duR2s = cur.duR2; dvR1s = dvR1; dvR2s = cur.dvR2;
        }
        if (first) { vL1s = vL1; vL2s = cur.vL2; dvL1s = dvL1; dvL2s = cur.dvL2; }

        // cell row i+1: grounded fraction, surface, slope factor, eta*H and its tangent
        const T gp = sigmoid(bedp + rr * Hp, p.sig_c);
        const T Sp = M<T>::max(bedp, -rr * Hp) + Hp;
        const T kHp = slope(Hp, bedp);
        T etaHp, detaHp;
        {
            EtaIn<T> a, da;
            a.ul = uL1;   a.ur = uR1s;  a.vt = v1;    a.vb = cur.v2;
            a.u_tl = uL0; a.u_tr = uR0s; a.u_bl = cur.uL2; a.u_br = uR2s;
            a.v_lt = vL1s; a.v_rt = vR1s; a.v_lb = vL2s; a.v_rb = vR2s;
            da.ul = duL1;   da.ur = duR1s;  da.vt = dv1;    da.vb = cur.dv2;
            da.u_tl = duL0; da.u_tr = duR0s; da.u_bl = cur.duL2; da.u_br = duR2s;
            da.v_lt = dvL1s; da.v_rt = dvR1s; da.v_lb = dvL2s; da.v_rb = dvR2s;
            const int ie = clampi(i + 1, 0, ny - 1);
            const EtaOut<T> e = cell_eta(a, Bp, ie, jcc, ny, nx, p);
            const T deta = cell_eta_tangent(e, da, Bp, ie, jcc, ny, nx, p);
            etaHp = e.eta * Hp;
            detaHp = deta * Hp + e.eta * dHp;
        }

        // stress tangents of row i and of vertex row i+1
        T dsxx, dsyy;
        {
            const NormalStress<T> s = normal_stress<T, true>(uL0, uR0s, v0, v1, etaH0, dxi, jc >= 0 && jc < nx);
            dsxx = s.d_ul * duL0 + s.d_ur * duR0s + s.d_vt * dv0 + s.d_vb * dv1 + s.d_etaH * detaH0;
        }
        {
            const NormalStress<T> s = normal_stress<T, false>(uL0, uR0s, v0, v1, etaH0, dxi, i >= 0 && i < ny);
            dsyy = s.d_ul * duL0 + s.d_ur * duR0s + s.d_vt * dv0 + s.d_vb * dv1 + s.d_etaH * detaH0;
        }
        T dsxy1;
        {
            const T etaH0L = __shfl_up_sync(FULL, etaH0, 1), etaHpL = __shfl_up_sync(FULL, etaHp, 1);
            const T detaH0L = __shfl_up_sync(FULL, detaH0, 1), detaHpL = __shfl_up_sync(FULL, detaHp, 1);
            const ShearStress<T> s = shear_stress(uL0, uL1, vL1s, v1, T(0.25) * (etaH0L + etaH0 + etaHpL + etaHp),
                                                  dxi, i + 1 > 0 && i + 1 < ny && jc > 0 && jc < nx);
            const T detaH = T(0.25) * (detaH0L + detaH0 + detaHpL + detaHp);
            dsxy1 = s.d_ut * duL0 + s.d_ub * duL1 + s.d_vl * dvL1s + s.d_vr * dv1 + s.d_etaH * detaH;
        }

        if (i >= i0) {  // warp-uniform
            const T dsxxL = __shfl_up_sync(FULL, dsxx, 1), dsxxR = __shfl_down_sync(FULL, dsxx, 1);
            const T dsxy0R = __shfl_down_sync(FULL, dsxy0, 1), dsxy1R = __shfl_down_sync(FULL, dsxy1, 1);
            const T HcL = __shfl_up_sync(FULL, Hc, 1), HcR = __shfl_down_sync(FULL, Hc, 1);
            const T dHcL = __shfl_up_sync(FULL, dHc, 1), dHcR = __shfl_down_sync(FULL, dHc, 1);
            const T gcL = __shfl_up_sync(FULL, gcc, 1), gcR = __shfl_down_sync(FULL, gcc, 1);
            const T ScL = __shfl_up_sync(FULL, Sc, 1), kHcL = __shfl_up_sync(FULL, kHc, 1);
            const T becL = __shfl_up_sync(FULL, bec, 1), becR = __shfl_down_sync(FULL, bec, 1);
            if (own) {
                const Ix ic = Ix(i) * nx + jc;
                // ---- mass row
                {
                    const T m = cur.m;
                    const Flux<T> ql = upwind_flux(uL0, HcL, Hc, jc > 0 && jc < nx);
                    const Flux<T> qr = upwind_flux(uR0s, Hc, HcR, jc + 1 > 0 && jc + 1 < nx);
                    const Flux<T> qt = upwind_flux(v0, Hc, Hm, i > 0 && i < ny);
                    const Flux<T> qb = upwind_flux(v1, Hp, Hc, i + 1 > 0 && i + 1 < ny);
                    const Calving<T> cv = calving_g(Hc, gcc, p);
                    T d = dHc / p.dt - cv.d_H * dHc;
                    d -= (ql.d_vel * duL0 + ql.d_Ha * dHcL + ql.d_Hb * dHc) * dxi;
                    d += (qr.d_vel * duR0s + qr.d_Ha * dHc + qr.d_Hb * dHcR) * dxi;
                    d += (qt.d_vel * dv0 + qt.d_Ha * dHc + qt.d_Hb * dHm) * dxi;
                    d -= (qb.d_vel * dv1 + qb.d_Ha * dHp + qb.d_Hb * dHc) * dxi;
                    const T jH = (T(1) - m) * d + m * dHc;
                    o_H[ic] = ADD ? cur.bH + jH : jH;
                }
                // ---- u-face (i, jc) and, at the right edge, (i, nx)
                {
                    T val = (dsxx - dsxxL) * dxi + (dsxy0 - dsxy1) * dxi;
                    const BasalDrag<T> tb = basal_drag_g(uL0, gcL, gcc, becL, bec, p);
                    val += tb.d_vel * duL0 + tb.d_H1 * dHcL + tb.d_H2 * dHc;
                    const T w = (jc > 0 && jc < nx) ? T(1) : T(0);   // driving: m = left, p = right
                    const T dS = Sc - ScL, Havg = T(0.5) * (HcL + Hc);
                    const T d_Hm = (T(0.5) * dS * dxi - Havg * kHcL * dxi) * w;
                    const T d_Hp = (T(0.5) * dS * dxi + Havg * kHc * dxi) * w;
                    val -= d_Hm * dHcL + d_Hp * dHc;
                    o_u[Ix(i) * (nx + 1) + jc] = ADD ? cur.bu + val : val;
                    if (jc == nx - 1) {
                        T ve = (dsxxR - dsxx) * dxi + (dsxy0R - dsxy1R) * dxi;
                        const BasalDrag<T> te = basal_drag_g(uR0s, gcc, gcR, bec, becR, p);
                        ve += te.d_vel * duR0s + te.d_H1 * dHc + te.d_H2 * dHcR;
                        const Ix oe = Ix(i) * (nx + 1) + nx;
                        o_u[oe] = ADD ? __ldg(base_u + oe) + ve : ve;
                    }
                }
                // ---- v-face (i, jc) and, at the bottom edge, (ny, jc)
                {
                    T val = (dsyym - dsyy) * dxi + (dsxy0R - dsxy0) * dxi;
                    const BasalDrag<T> tb = basal_drag_g(v0, gm, gcc, bem, bec, p);
                    val += tb.d_vel * dv0 + tb.d_H1 * dHm + tb.d_H2 * dHc;
                    const T w = (i > 0 && i < ny) ? T(1) : T(0);     // driving: m = bottom (row i), p = top
                    const T dS = Sm - Sc, Havg = T(0.5) * (Hc + Hm);
                    const T d_Hm = (T(0.5) * dS * dxi - Havg * kHc * dxi) * w;
                    const T d_Hp = (T(0.5) * dS * dxi + Havg * kHm * dxi) * w;
                    val -= d_Hm * dHc + d_Hp * dHm;
                    o_v[ic] = ADD ? cur.bv + val : val;
                    if (i == ny - 1) {
                        T ve = (dsyy - T(0)) * dxi + (dsxy1R - dsxy1) * dxi;
                        const BasalDrag<T> te = basal_drag_g(v1, gcc, gp, bec, betap, p);
                        ve += te.d_vel * dv1 + te.d_H1 * dHc + te.d_H2 * dHp;
                        const Ix oe = Ix(ny) * nx + jc;
                        o_v[oe] = ADD ? __ldg(base_v + oe) + ve : ve;
                    }
                }
            }
        }
        // roll the window one row down
        dsyym = dsyy; dsxy0 = dsxy1; etaH0 = etaHp; detaH0 = detaHp;
        Hm = Hc; gm = gcc; Sm = Sc; bem = bec; kHm = kHc; dHm = dHc;
        Hc = Hp; gcc = gp; Sc = Sp; bec = betap; kHc = kHp; dHc = dHp;
        uL0 = uL1; uL1 = cur.uL2; uR0 = uR1; uR1 = cur.uR2;
        v0 = v1; v1 = cur.v2; vL1 = cur.vL2; vR1 = cur.vR2;
        duL0 = duL1; duL1 = cur.duL2; duR0 = duR1; duR1 = cur.duR2;
        dv0 = dv1; dv1 = cur.dv2; dvL1 = cur.dvL2; dvR1 = cur.dvR2;
    }
}

// --------------------------------------------------------------------------
// VJP lambda^T J, streaming form (what launch_vjp runs): the warp-strip march
// of jvp_stream_kernel with lambda as the direction.  The velocity-velocity
// block is applied as the forward tangent (the viscous block is symmetric,
// glide/cuda/residuals.cu:709); the H rows gather, per cell, the transposed
// flux, drag and driving partials of its four faces, the eta*H partials of
// its normal stresses and the vertex weights of its four corner shear
// stresses.  At iteration i the kernel forms the cell row i+1, the stress
// tangents of row i and of vertex row i+1, the vertex weights of row i+1 and
// the H-row contributions of v-face row i+1; the rows above come from the
// previous iterations (glide/cuda/residuals.cu:586-1023).  exact_boundary = 0
// drops the contributions the reference drops at clamped boundary reads (only
// non-zero with gl_derivatives), 1 keeps them.  With RF the output is
// f - lambda^T J.
// --------------------------------------------------------------------------
// 128-thread CTAs: with 150-180 registers per thread three fit on an SM in
// FP32 (12 warps; one 256-thread CTA would give 8), two in FP64
constexpr int VS_NT = 128;
#ifndef GLIDE_VS_MINB32
#define GLIDE_VS_MINB32 3
#endif
#ifndef GLIDE_VS_MINB64
#define GLIDE_VS_MINB64 2
#endif
template <typename T, bool RF, typename Ix>
__global__ void __launch_bounds__(VS_NT, sizeof(T) == 4 ? GLIDE_VS_MINB32 : GLIDE_VS_MINB64) vjp_stream_kernel(
    T* __restrict__ o_u, T* __restrict__ o_v, T* __restrict__ o_H,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ H,
    const T* __restrict__ lu, const T* __restrict__ lv, const T* __restrict__ lH,
    const T* __restrict__ bed, const T* __restrict__ B, const T* __restrict__ beta, const T* __restrict__ mask,
    const T* __restrict__ f_u, const T* __restrict__ f_v, const T* __restrict__ f_H, int exact_boundary, Geo g,
    Phys<T> p, int n_strips, int rows, int n_warps) {
    const int ny = g.ny, nx = g.nx;
    const int wid = blockIdx.x * (VS_NT / 32) + threadIdx.x / 32;
    if (wid >= n_warps) return;  // whole warp
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.y;
    u += b * g.nu(); v += b * g.nv(); H += b * g.nc();
    lu += b * g.nu(); lv += b * g.nv(); lH += b * g.nc();
    if constexpr (RF) { f_u += b * g.nu(); f_v += b * g.nv(); f_H += b * g.nc(); }
    bed += b * g.nc(); B += b * g.nc(); beta += b * g.nc(); mask += b * g.nc();
    o_u += b * g.nu(); o_v += b * g.nv(); o_H += b * g.nc();

    const int strip = wid % n_strips, chunk = wid / n_strips;
    const int i0 = chunk * rows;
    const int i1 = min(i0 + rows, ny);
    const int jc = strip * SW - 1 + lane;
    const int jcc = clampi(jc, 0, nx - 1);
    const int juL = clampi(jc, 0, nx);
    const int juR = clampi(jc + 1, 0, nx);
    const int jvL = clampi(jc - 1, 0, nx - 1), jvR = clampi(jc + 1, 0, nx - 1);
    const bool first = lane == 0, last = lane == 31;
    const bool own = lane >= 1 && lane <= SW && jc < nx;
    const unsigned FULL = 0xffffffffu;
    const T dxi = p.dxi;
    const T rr = rho_ratio<T>();
    auto Uf = [&](const T* a, int r, int col) -> T {
        return __ldg(a + Ix(clampi(r, 0, ny - 1)) * (nx + 1) + col);
    };
    auto Vf = [&](const T* a, int r, int col) -> T { return __ldg(a + Ix(clampi(r, 0, ny)) * nx + col); };
    auto Cell = [&](const T* a, int r) -> T { return __ldg(a + Ix(clampi(r, 0, ny - 1)) * nx + jcc); };
    auto slope = [&](T Hx, T bx) -> T { return T(1) + (bx > -rr * Hx ? T(0) : -rr); };

    int i = i0 - 2;
    T uL0 = Uf(u, i, juL), uL1 = Uf(u, i + 1, juL);
    T uR0 = last ? Uf(u, i, juR) : T(0), uR1 = last ? Uf(u, i + 1, juR) : T(0);
    T v0 = Vf(v, i, jcc), v1 = Vf(v, i + 1, jcc);
    T vL1 = first ? Vf(v, i + 1, jvL) : T(0), vR1 = last ? Vf(v, i + 1, jvR) : T(0);
    T luL0 = Uf(lu, i, juL), luL1 = Uf(lu, i + 1, juL);
    T luR0 = last ? Uf(lu, i, juR) : T(0), luR1 = last ? Uf(lu, i + 1, juR) : T(0);
    T lv0 = Vf(lv, i, jcc), lv1 = Vf(lv, i + 1, jcc);
    T lvL1 = first ? Vf(lv, i + 1, jvL) : T(0), lvR1 = last ? Vf(lv, i + 1, jvR) : T(0);
    // cell rows m = i-1 and c = i: thickness, grounded fraction, surface, beta,
    // slope factor, masked lambda_H; row c also its mask and lambda_H
    T Hm = T(0), gm = T(0), Sm = T(0), bem = T(0), kHm = T(0), ltm = T(0);
    T Hc = T(0), gcc = T(0), Sc = T(0), bec = T(0), kHc = T(0), ltc = T(0), mc = T(0), lHc = T(0);
    // eta, eta*H and the tangent of eta*H of row i; stress tangents of row i-1
    // (syy) and vertex row i (sxy); vertex weights of row i; H-row terms of
    // v-face row i
    T eta0 = T(0), etaH0 = T(0), detaH0 = T(0), dsxy0 = T(0), dsyym = T(0), W0 = T(0), CvT0 = T(0), CvB0 = T(0);
    constexpr bool PREFETCH = sizeof(T) == 4;
    const int jo = jc < nx ? (jc < 0 ? 0 : jc) : nx - 1;
    struct RowIn {
        T uL2, uR2, v2, vL2, vR2, luL2, luR2, lv2, lvL2, lvR2, H, bed, beta, B, lH, m, fu, fv, fH;
    };
    auto load_row = [&](int k) {
        RowIn r;
        r.uL2 = Uf(u, k + 2, juL);
        r.uR2 = last ? Uf(u, k + 2, juR) : T(0);
        r.v2 = Vf(v, k + 2, jcc);
        r.vL2 = first ? Vf(v, k + 2, jvL) : T(0);
        r.vR2 = last ? Vf(v, k + 2, jvR) : T(0);
        r.luL2 = Uf(lu, k + 2, juL);
        r.luR2 = last ? Uf(lu, k + 2, juR) : T(0);
        r.lv2 = Vf(lv, k + 2, jcc);
        r.lvL2 = first ? Vf(lv, k + 2, jvL) : T(0);
        r.lvR2 = last ? Vf(lv, k + 2, jvR) : T(0);
        r.H = Cell(H, k + 1); r.bed = Cell(bed, k + 1); r.beta = Cell(beta, k + 1); r.B = Cell(B, k + 1);
        r.lH = Cell(lH, k + 1); r.m = Cell(mask, k + 1);
        if constexpr (RF) {
            const Ix ro = clampi(k, 0, ny - 1);
            r.fu = __ldg(f_u + ro * (nx + 1) + jo);
            r.fv = __ldg(f_v + ro * nx + jo);
            r.fH = __ldg(f_H + ro * nx + jo);
        } else {
            r.fu = r.fv = r.fH = T(0);
        }
        return r;
    };
    RowIn nxt;
    if constexpr (PREFETCH) nxt = load_row(i);
    for (; i < i1; ++i) {
        RowIn cur;
        if constexpr (PREFETCH) {
            cur = nxt;
            nxt = load_row(i + 1);
        } else {
            cur = load_row(i);
        }
        const T Hp = cur.H, bedp = cur.bed, betap = cur.beta, Bp = cur.B;
        const T mp = cur.m, lHp = cur.lH;

        T uR0s = __shfl_down_sync(FULL, uL0, 1), uR1s = __shfl_down_sync(FULL, uL1, 1);
        T uR2s = __shfl_down_sync(FULL, cur.uL2, 1);
        T vL1s = __shfl_up_sync(FULL, v1, 1), vL2s = __shfl_up_sync(FULL, cur.v2, 1);
        T vR1s = __shfl_down_sync(FULL, v1, 1), vR2s = __shfl_down_sync(FULL, cur.v2, 1);
        T luR0s = __shfl_down_sync(FULL, luL0, 1), luR1s = __shfl_down_sync(FULL, luL1, 1);
        T luR2s = __shfl_down_sync(FULL, cur.luL2, 1);
        T lvL1s = __shfl_up_sync(FULL, lv1, 1), lvL2s = __shfl_up_sync(FULL, cur.lv2, 1);
        T lvR1s = __shfl_down_sync(FULL, lv1, 1), lvR2s = __shfl_down_sync(FULL, cur.lv2, 1);
        if (last) {
            uR0s = uR0; uR1s = uR1; uR2s = cur.uR2; vR1s = vR1; vR2s = cur.vR2;
            luR0s = luR0; luR1s = luR1; luR2s = cur.luR2; lvR1s = lvR1; lvR2s = cur.lvR2;
        }
        if (first) { vL1s = vL1; vL2s = cur.vL2; lvL1s = lvL1; lvL2s = cur.lvL2; }

        // cell row i+1
        const T gp = sigmoid(bedp + rr * Hp, p.sig_c);
        const T Sp = M<T>::max(bedp, -rr * Hp) + Hp;
        const T kHp = slope(Hp, bedp);
        const T ltp = lHp * (T(1) - mp);
        T etaP, etaHp, detaHp;
        {
            EtaIn<T> a, da;
            a.ul = uL1;   a.ur = uR1s;  a.vt = v1;    a.vb = cur.v2;
            a.u_tl = uL0; a.u_tr = uR0s; a.u_bl = cur.uL2; a.u_br = uR2s;
            a.v_lt = vL1s; a.v_rt = vR1s; a.v_lb = vL2s; a.v_rb = vR2s;
            da.ul = luL1;   da.ur = luR1s;  da.vt = lv1;    da.vb = cur.lv2;
            da.u_tl = luL0; da.u_tr = luR0s; da.u_bl = cur.luL2; da.u_br = luR2s;
            da.v_lt = lvL1s; da.v_rt = lvR1s; da.v_lb = lvL2s; da.v_rb = lvR2s;
            const int ie = clampi(i + 1, 0, ny - 1);
            const EtaOut<T> e = cell_eta(a, Bp, ie, jcc, ny, nx, p);
            const T deta = cell_eta_tangent(e, da, Bp, ie, jcc, ny, nx, p);
            etaP = e.eta;
            etaHp = e.eta * Hp;
            detaHp = deta * Hp;
        }

        // stress tangents of row i, vertex row i+1 (with its H-row weight)
        T dsxx, dsyy, hx, hy;
        {
            const NormalStress<T> s = normal_stress<T, true>(uL0, uR0s, v0, v1, etaH0, dxi, jc >= 0 && jc < nx);
            dsxx = s.d_ul * luL0 + s.d_ur * luR0s + s.d_vt * lv0 + s.d_vb * lv1 + s.d_etaH * detaH0;
            hx = s.d_etaH;
        }
        {
            const NormalStress<T> s = normal_stress<T, false>(uL0, uR0s, v0, v1, etaH0, dxi, i >= 0 && i < ny);
            dsyy = s.d_ul * luL0 + s.d_ur * luR0s + s.d_vt * lv0 + s.d_vb * lv1 + s.d_etaH * detaH0;
            hy = s.d_etaH;
        }
        T dsxy1, W1;
        {
            const T etaH0L = __shfl_up_sync(FULL, etaH0, 1), etaHpL = __shfl_up_sync(FULL, etaHp, 1);
            const T detaH0L = __shfl_up_sync(FULL, detaH0, 1), detaHpL = __shfl_up_sync(FULL, detaHp, 1);
            const bool valid = i + 1 > 0 && i + 1 < ny && jc > 0 && jc < nx;
            const ShearStress<T> s = shear_stress(uL0, uL1, vL1s, v1, T(0.25) * (etaH0L + etaH0 + etaHpL + etaHp),
                                                  dxi, valid);
            const T detaH = T(0.25) * (detaH0L + detaH0 + detaHpL + detaHp);
            dsxy1 = s.d_ut * luL0 + s.d_ub * luL1 + s.d_vl * lvL1s + s.d_vr * lv1 + s.d_etaH * detaH;
            const T w = valid ? (luL1 - luL0 - lv1 + lvL1s) * dxi : T(0);
            W1 = w * s.d_etaH * T(0.25);
        }
        // H-row terms of v-face row i+1 (top cell: row i, bottom cell: row i+1)
        T CvT1, CvB1;
        {
            const bool valid = i + 1 > 0 && i + 1 < ny;
            const Flux<T> q = upwind_flux(v1, Hp, Hc, valid);
            const T a = (ltp - ltc) * dxi;
            const BasalDrag<T> tb = basal_drag_g(v1, gcc, gp, bec, betap, p);
            const T w = valid ? T(1) : T(0);     // driving: m = bottom (row i+1), p = top (row i)
            const T dS = Sc - Sp, Havg = T(0.5) * (Hp + Hc);
            const T d_Hm = (T(0.5) * dS * dxi - Havg * kHp * dxi) * w;
            const T d_Hp = (T(0.5) * dS * dxi + Havg * kHc * dxi) * w;
            CvT1 = a * q.d_Hb + lv1 * (tb.d_H1 - d_Hp);
            CvB1 = a * q.d_Ha + lv1 * (tb.d_H2 - d_Hm);
        }

        if (i >= i0) {  // warp-uniform
            const T HcL = __shfl_up_sync(FULL, Hc, 1);
            const T gcL = __shfl_up_sync(FULL, gcc, 1), gcR = __shfl_down_sync(FULL, gcc, 1);
            const T ScL = __shfl_up_sync(FULL, Sc, 1), kHcL = __shfl_up_sync(FULL, kHc, 1);
            const T becL = __shfl_up_sync(FULL, bec, 1), becR = __shfl_down_sync(FULL, bec, 1);
            const T ltL = __shfl_up_sync(FULL, ltc, 1);
            // H-row terms of u-face (i, jc) (left cell: jc-1, right cell: jc)
            T CuL, CuR;
            {
                const bool valid = jc > 0 && jc < nx;
                const Flux<T> q = upwind_flux(uL0, HcL, Hc, valid);
                const T a = (ltL - ltc) * dxi;
                const BasalDrag<T> tb = basal_drag_g(uL0, gcL, gcc, becL, bec, p);
                const T w = valid ? T(1) : T(0);  // driving: m = left, p = right
                const T dS = Sc - ScL, Havg = T(0.5) * (HcL + Hc);
                const T d_Hm = (T(0.5) * dS * dxi - Havg * kHcL * dxi) * w;
                const T d_Hp = (T(0.5) * dS * dxi + Havg * kHc * dxi) * w;
                CuL = a * q.d_Ha + luL0 * (tb.d_H1 - d_Hm);
                CuR = a * q.d_Hb + luL0 * (tb.d_H2 - d_Hp);
            }
            const T CuLR = __shfl_down_sync(FULL, CuL, 1), CuRR = __shfl_down_sync(FULL, CuR, 1);
            const T dsxxL = __shfl_up_sync(FULL, dsxx, 1), dsxxR = __shfl_down_sync(FULL, dsxx, 1);
            const T dsxy0R = __shfl_down_sync(FULL, dsxy0, 1), dsxy1R = __shfl_down_sync(FULL, dsxy1, 1);
            const T W0R = __shfl_down_sync(FULL, W0, 1), W1R = __shfl_down_sync(FULL, W1, 1);
            const T ltR = __shfl_down_sync(FULL, ltc, 1);
            if (own) {
                const Ix ic = Ix(i) * nx + jc;
                // ---- H row
                {
                    const Calving<T> cv = calving_g(Hc, gcc, p);
                    T acc = ltc / p.dt - ltc * cv.d_H;
                    acc += CuR + CuLR + CvB0 + CvT1;
                    if (exact_boundary) {
                        if (jc == 0) acc += CuL;
                        if (jc == nx - 1) acc += CuRR;
                        if (i == 0) acc += CvT0;
                        if (i == ny - 1) acc += CvB1;
                    }
                    acc += (luL0 - luR0s) * hx * eta0 * dxi;
                    acc += (lv1 - lv0) * hy * eta0 * dxi;
                    acc += eta0 * (W0 + W0R + W1 + W1R);
                    acc += lHc * mc;
                    o_H[ic] = RF ? cur.fH - acc : acc;
                }
                // ---- u-face (i, jc) and, at the right edge, (i, nx)
                {
                    T val = (dsxx - dsxxL) * dxi + (dsxy0 - dsxy1) * dxi;
                    const BasalDrag<T> tb = basal_drag_g(uL0, gcL, gcc, becL, bec, p);
                    const Flux<T> q = upwind_flux(uL0, HcL, Hc, jc > 0 && jc < nx);
                    val += luL0 * tb.d_vel + (ltL - ltc) * dxi * q.d_vel;
                    o_u[Ix(i) * (nx + 1) + jc] = RF ? cur.fu - val : val;
                    if (jc == nx - 1) {
                        T ve = (dsxxR - dsxx) * dxi + (dsxy0R - dsxy1R) * dxi;
                        const BasalDrag<T> te = basal_drag_g(uR0s, gcc, gcR, bec, becR, p);
                        const Flux<T> qe = upwind_flux(uR0s, Hc, Hc, false);  // H(i, nx) clamps to H(i, nx-1)
                        ve += luR0s * te.d_vel + (ltc - ltR) * dxi * qe.d_vel;
                        const Ix oe = Ix(i) * (nx + 1) + nx;
                        o_u[oe] = RF ? __ldg(f_u + oe) - ve : ve;
                    }
                }
                // ---- v-face (i, jc) and, at the bottom edge, (ny, jc)
                {
                    T val = (dsyym - dsyy) * dxi + (dsxy0R - dsxy0) * dxi;
                    const BasalDrag<T> tb = basal_drag_g(v0, gm, gcc, bem, bec, p);
                    const Flux<T> q = upwind_flux(v0, Hc, Hm, i > 0 && i < ny);
                    val += lv0 * tb.d_vel + (ltc - ltm) * dxi * q.d_vel;
                    o_v[ic] = RF ? cur.fv - val : val;
                    if (i == ny - 1) {
                        T ve = (dsyy - T(0)) * dxi + (dsxy1R - dsxy1) * dxi;
                        const BasalDrag<T> te = basal_drag_g(v1, gcc, gp, bec, betap, p);
                        const Flux<T> qe = upwind_flux(v1, Hp, Hc, false);
                        ve += lv1 * te.d_vel + (ltp - ltc) * dxi * qe.d_vel;
                        const Ix oe = Ix(ny) * nx + jc;
                        o_v[oe] = RF ? __ldg(f_v + oe) - ve : ve;
                    }
                }
            }
        }
        // roll the window one row down
        dsyym = dsyy; dsxy0 = dsxy1; W0 = W1; CvT0 = CvT1; CvB0 = CvB1;
        eta0 = etaP; etaH0 = etaHp; detaH0 = detaHp;
        Hm = Hc; gm = gcc; Sm = Sc; bem = bec; kHm = kHc; ltm = ltc;
        Hc = Hp; gcc = gp; Sc = Sp; bec = betap; kHc = kHp; ltc = ltp; mc = mp; lHc = lHp;
        uL0 = uL1; uL1 = cur.uL2; uR0 = uR1; uR1 = cur.uR2;
        v0 = v1; v1 = cur.v2; vL1 = cur.vL2; vR1 = cur.vR2;
        luL0 = luL1; luL1 = cur.luL2; luR0 = luR1; luR1 = cur.luR2;
        lv0 = lv1; lv1 = cur.lv2; lvL1 = cur.lvL2; lvR1 = cur.lvR2;
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

// strips of SW columns, row chunks sized for ~32 warps per SM
struct StreamShape {
    int n_strips, rows, n_warps;
};
// 32-bit element offsets suffice when every field of one problem has fewer
// than 2^31 elements (u and v have (ny+1)(nx+1) at most)
static inline bool index32(const Geo& g) { return int64_t(g.ny + 1) * (g.nx + 1) < (int64_t(1) << 31); }

static inline StreamShape stream_shape(const Geo& g) {
    StreamShape sh;
    sh.n_strips = (g.nx + SW - 1) / SW;
    int rows = int((int64_t(g.ny) * sh.n_strips * g.nb + 148 * 32 - 1) / (148 * 32));
    sh.rows = rows < 8 ? 8 : (rows > 128 ? 128 : rows);
    sh.n_warps = sh.n_strips * ((g.ny + sh.rows - 1) / sh.rows);
    return sh;
}

template <typename T>
int launch_residual(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, void* r_u, void* r_v,
                    void* r_H, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    const StreamShape sh = stream_shape(g);
    const dim3 grid((sh.n_warps + 7) / 8, g.nb);
    auto go = [&](auto kernel) {
        glide::count_launch(), kernel<<<grid, 256, 0, s>>>(
            (T*)r_u, (T*)r_v, (T*)r_H, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)f_u,
            (const T*)f_v, (const T*)f_H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->mask,
            (const T*)a->gamma, g, p, sh.n_strips, sh.rows, sh.n_warps);
    };
    if (index32(g))
        go(residual_stream_kernel<T, int>);
    else
        go(residual_stream_kernel<T, int64_t>);
    return (int)cudaGetLastError();
}

// j = J(U) d, or j = base + J(U) d when base_u is not null
template <typename T>
int launch_jvp(const GlideLevelArgs* a, const void* d_u, const void* d_v, const void* d_H, const void* base_u,
               const void* base_v, const void* base_H, void* j_u, void* j_v, void* j_H, cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    const StreamShape sh = stream_shape(g);
    const dim3 grid((sh.n_warps + 7) / 8, g.nb);
    auto go = [&](auto kernel) {
        glide::count_launch(), kernel<<<grid, 256, 0, s>>>(
            (T*)j_u, (T*)j_v, (T*)j_H, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)d_u,
            (const T*)d_v, (const T*)d_H, (const T*)base_u, (const T*)base_v, (const T*)base_H, (const T*)a->bed,
            (const T*)a->B, (const T*)a->beta, (const T*)a->mask, g, p, sh.n_strips, sh.rows, sh.n_warps);
    };
    const bool i32 = index32(g);
    if (base_u)
        i32 ? go(jvp_stream_kernel<T, true, int>) : go(jvp_stream_kernel<T, true, int64_t>);
    else
        i32 ? go(jvp_stream_kernel<T, false, int>) : go(jvp_stream_kernel<T, false, int64_t>);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_vjp(const GlideLevelArgs* a, const void* l_u, const void* l_v, const void* l_H, const void* f_u,
               const void* f_v, const void* f_H, void* o_u, void* o_v, void* o_H, int exact_boundary,
               cudaStream_t s) {
    Geo g{a->ny, a->nx, a->nb};
    Phys<T> p = make_phys<T>(a->params, a->dx, a->dt);
    const StreamShape sh = stream_shape(g);
    const dim3 grid((sh.n_warps + VS_NT / 32 - 1) / (VS_NT / 32), g.nb);
    auto go = [&](auto kernel) {
        glide::count_launch(), kernel<<<grid, VS_NT, 0, s>>>(
            (T*)o_u, (T*)o_v, (T*)o_H, (const T*)a->u, (const T*)a->v, (const T*)a->H, (const T*)l_u,
            (const T*)l_v, (const T*)l_H, (const T*)a->bed, (const T*)a->B, (const T*)a->beta, (const T*)a->mask,
            (const T*)f_u, (const T*)f_v, (const T*)f_H, exact_boundary, g, p, sh.n_strips, sh.rows, sh.n_warps);
    };
    const bool i32 = index32(g);
    if (f_u != nullptr)
        i32 ? go(vjp_stream_kernel<T, true, int>) : go(vjp_stream_kernel<T, true, int64_t>);
    else
        i32 ? go(vjp_stream_kernel<T, false, int>) : go(vjp_stream_kernel<T, false, int64_t>);
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
template int launch_jvp<float>(const GlideLevelArgs*, const void*, const void*, const void*, const void*,
                               const void*, const void*, void*, void*, void*, cudaStream_t);
template int launch_jvp<double>(const GlideLevelArgs*, const void*, const void*, const void*, const void*,
                                const void*, const void*, void*, void*, void*, cudaStream_t);
template int launch_vjp<float>(const GlideLevelArgs*, const void*, const void*, const void*, const void*, const void*,
                               const void*, void*, void*, void*, int, cudaStream_t);
template int launch_vjp<double>(const GlideLevelArgs*, const void*, const void*, const void*, const void*,
                                const void*, const void*, void*, void*, void*, int, cudaStream_t);
template int launch_grad_beta<float>(const GlideLevelArgs*, const void*, const void*, void*, int, cudaStream_t);
template int launch_grad_beta<double>(const GlideLevelArgs*, const void*, const void*, void*, int, cudaStream_t);

}  // namespace glide
