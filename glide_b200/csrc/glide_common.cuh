// Shared device code for the SSA hot path on B200 (sm_100a).
//
// Physics follows the reference discretisation (glide/cuda/stress.cu,
// glide/cuda/flux.cu, glide/cuda/viscosity.cu); every term returns its value
// together with the partial derivatives the solvers need, written as plain
// value-plus-partials structs instead of the reference's dual numbers.
// Everything is templated on the working precision T (float or double).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "glide_b200.h"

namespace glide {

// host-side count of kernel launches issued by this library (also counts
// launches recorded during stream capture); see glide_launch_count
void count_launch();
long long launch_total();

// --------------------------------------------------------------------------
// precision helpers
// --------------------------------------------------------------------------
template <typename T> struct M;
// FP32 exp/pow: the hardware approximations by default, as the reference's
// --use_fast_math build of its ice kernels uses (glide/kernels.py:72);
// -DGLIDE_FP32_ACCURATE_MATH=1 selects expf/powf and IEEE division.
#ifndef GLIDE_FP32_ACCURATE_MATH
#define GLIDE_FP32_ACCURATE_MATH 0
#endif
template <> struct M<float> {
#if GLIDE_FP32_ACCURATE_MATH
    static __device__ __forceinline__ float exp(float x) { return expf(x); }
    static __device__ __forceinline__ float pow(float x, float y) { return powf(x, y); }
    static __device__ __forceinline__ float rcp(float x) { return 1.0f / x; }
#else
    static __device__ __forceinline__ float exp(float x) { return __expf(x); }
    static __device__ __forceinline__ float pow(float x, float y) { return __powf(x, y); }
    // reciprocal of the LU pivots and of the sigmoid denominator: the fast
    // approximate division, as the reference's fast-math build divides
    static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
#endif
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float abs(float x) { return fabsf(x); }
    static __device__ __forceinline__ float copysign(float a, float b) { return copysignf(a, b); }
    static __device__ __forceinline__ float max(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float min(float a, float b) { return fminf(a, b); }
};
template <> struct M<double> {
    static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
    static __device__ __forceinline__ double pow(double x, double y) { return ::pow(x, y); }
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double abs(double x) { return fabs(x); }
    static __device__ __forceinline__ double copysign(double a, double b) { return ::copysign(a, b); }
    static __device__ __forceinline__ double max(double a, double b) { return fmax(a, b); }
    static __device__ __forceinline__ double min(double a, double b) { return fmin(a, b); }
};

// rho_ice / rho_water, as in glide/cuda/stress.cu:250
template <typename T> __device__ __forceinline__ T rho_ratio() { return T(0.917); }

// Physical parameters converted to the working precision.
template <typename T> struct Phys {
    T glen_exp;      // (1-n)/(2n)
    T eps_reg, water_drag, calving_rate, sig_c;
    int gl_deriv;
    T dx, dxi, dt;
};

template <typename T>
inline Phys<T> make_phys(const GlidePhysicsParams& p, double dx, double dt) {
    Phys<T> q;
    T n = T(p.n);
    q.glen_exp = (T(1) - n) / (T(2) * n);
    q.eps_reg = T(p.eps_reg);
    q.water_drag = T(p.water_drag);
    q.calving_rate = T(p.calving_rate);
    q.sig_c = T(p.gl_sigmoid_c);
    q.gl_deriv = p.gl_derivatives;
    q.dx = T(dx);
    q.dxi = T(1) / T(dx);
    q.dt = T(dt);
    return q;
}

// Geometry of one level (batch of nb independent problems).
struct Geo {
    int ny, nx, nb;
    __host__ __device__ int64_t nu() const { return int64_t(ny) * (nx + 1); }
    __host__ __device__ int64_t nv() const { return int64_t(ny + 1) * nx; }
    __host__ __device__ int64_t nc() const { return int64_t(ny) * nx; }
};

__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

// --------------------------------------------------------------------------
// clamped global accessors (same semantics as glide/cuda/common.cu:78-125:
// every index is clamped to the field's own extent).  Offsets are 32-bit
// element counts: the entry points reject problems whose fields reach 2^31
// elements (GLIDE_E_TOO_LARGE).
// --------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T ldu(const T* __restrict__ u, int i, int j, int ny, int nx) {
    return __ldg(u + (clampi(i, 0, ny - 1) * (nx + 1) + clampi(j, 0, nx)));
}
template <typename T>
__device__ __forceinline__ T ldv(const T* __restrict__ v, int i, int j, int ny, int nx) {
    return __ldg(v + (clampi(i, 0, ny) * nx + clampi(j, 0, nx - 1)));
}
template <typename T>
__device__ __forceinline__ T ldc(const T* __restrict__ a, int i, int j, int ny, int nx) {
    return __ldg(a + (clampi(i, 0, ny - 1) * nx + clampi(j, 0, nx - 1)));
}

// Stage a clamped window [r0, r0+R) x [c0, c0+C) of a (rows x cols) field
// into shared memory (row-major, leading dimension C).
template <typename T>
__device__ __forceinline__ void stage(T* __restrict__ s, const T* __restrict__ g, int rows, int cols, int r0,
                                      int c0, int R, int C, int tid, int nthreads) {
    for (int k = tid; k < R * C; k += nthreads) {
        int r = k / C, c = k - r * C;
        int gi = clampi(r0 + r, 0, rows - 1), gj = clampi(c0 + c, 0, cols - 1);
        s[k] = __ldg(g + int64_t(gi) * cols + gj);
    }
}

// --------------------------------------------------------------------------
// local terms (value + partials)
// --------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T sigmoid(T z, T c) {
    T s = M<T>::min(M<T>::max(c * z, T(-20)), T(20));   // common.cu:67-70
    return M<T>::rcp(T(1) + M<T>::exp(-s));
}

// Normal stress on a cell (stress.cu:43-102).  XX: 2 etaH (2 ux + vy);
// YY: 2 etaH (ux + 2 vy).  Zero when the cell is outside the domain.
template <typename T> struct NormalStress {
    T res, d_ul, d_ur, d_vt, d_vb, d_etaH;
};
template <typename T, bool XX>
__device__ __forceinline__ NormalStress<T> normal_stress(T ul, T ur, T vt, T vb, T etaH, T dxi, bool valid) {
    NormalStress<T> o;
    T pre = T(2) * etaH * dxi;
    T e = XX ? (T(2) * (ur - ul) * dxi + (vt - vb) * dxi) : ((ur - ul) * dxi + T(2) * (vt - vb) * dxi);
    T w = valid ? T(1) : T(0);
    o.res = T(2) * etaH * e * w;
    o.d_ul = (XX ? T(-2) : T(-1)) * pre * w;
    o.d_ur = (XX ? T(2) : T(1)) * pre * w;
    o.d_vt = (XX ? T(1) : T(2)) * pre * w;
    o.d_vb = (XX ? T(-1) : T(-2)) * pre * w;
    o.d_etaH = T(2) * e * w;
    return o;
}

// Shear stress on a vertex (stress.cu:159-183): 2 etaH eps_xy, zero on boundary vertices.
template <typename T> struct ShearStress {
    T res, d_ut, d_ub, d_vl, d_vr, d_etaH;
};
template <typename T>
__device__ __forceinline__ ShearStress<T> shear_stress(T ut, T ub, T vl, T vr, T etaH, T dxi, bool valid) {
    ShearStress<T> o;
    T w = valid ? T(1) : T(0);
    T exy = T(0.5) * ((ut - ub) * dxi + (vr - vl) * dxi);
    T pre = etaH * dxi * w;
    o.res = T(2) * etaH * exy * w;
    o.d_ut = pre;
    o.d_ub = -pre;
    o.d_vl = -pre;
    o.d_vr = pre;
    o.d_etaH = T(2) * exy * w;
    return o;
}

// Basal drag between cells 1 and 2 of a face (stress.cu:244-276, :330-361).
template <typename T> struct BasalDrag {
    T res, d_vel, d_H1, d_H2, d_beta1, d_beta2;
};
template <typename T>
__device__ __forceinline__ BasalDrag<T> basal_drag(T vel, T H1, T H2, T bed1, T bed2, T beta1, T beta2,
                                                   const Phys<T>& p) {
    BasalDrag<T> o;
    T z1 = bed1 + rho_ratio<T>() * H1, z2 = bed2 + rho_ratio<T>() * H2;
    T g1 = sigmoid(z1, p.sig_c), g2 = sigmoid(z2, p.sig_c);
    T be = T(0.5) * ((g1 * beta1 + (T(1) - g1) * p.water_drag) + (g2 * beta2 + (T(1) - g2) * p.water_drag));
    o.res = -be * vel;
    o.d_vel = -be;
    o.d_beta1 = T(-0.5) * g1 * vel;
    o.d_beta2 = T(-0.5) * g2 * vel;
    if (p.gl_deriv) {
        T s1 = p.sig_c * g1 * (T(1) - g1), s2 = p.sig_c * g2 * (T(1) - g2);
        o.d_H1 = T(-0.5) * (rho_ratio<T>() * s1) * (beta1 - p.water_drag) * vel;
        o.d_H2 = T(-0.5) * (rho_ratio<T>() * s2) * (beta2 - p.water_drag) * vel;
    } else {
        o.d_H1 = T(0);
        o.d_H2 = T(0);
    }
    return o;
}

// Same drag with the two grounded fractions already known (the Vanka loop
// hoists the neighbour's sigmoid out of its Newton iterations).
template <typename T>
__device__ __forceinline__ BasalDrag<T> basal_drag_g(T vel, T g1, T g2, T beta1, T beta2, const Phys<T>& p) {
    BasalDrag<T> o;
    T be = T(0.5) * ((g1 * beta1 + (T(1) - g1) * p.water_drag) + (g2 * beta2 + (T(1) - g2) * p.water_drag));
    o.res = -be * vel;
    o.d_vel = -be;
    o.d_beta1 = T(-0.5) * g1 * vel;
    o.d_beta2 = T(-0.5) * g2 * vel;
    o.d_H1 = T(0);
    o.d_H2 = T(0);
    if (p.gl_deriv) {
        T s1 = p.sig_c * g1 * (T(1) - g1), s2 = p.sig_c * g2 * (T(1) - g2);
        o.d_H1 = T(-0.5) * (rho_ratio<T>() * s1) * (beta1 - p.water_drag) * vel;
        o.d_H2 = T(-0.5) * (rho_ratio<T>() * s2) * (beta2 - p.water_drag) * vel;
    }
    return o;
}

// Driving stress H_avg (S_p - S_m)/dx on a face (stress.cu:406-436, :481-510);
// x-faces: m = left, p = right; y-faces: m = bottom (row i), p = top (row i-1).
template <typename T> struct Driving {
    T res, d_Hm, d_Hp;
};
template <typename T>
__device__ __forceinline__ Driving<T> driving(T Hm, T Hp, T bedm, T bedp, T dxi, bool valid) {
    Driving<T> o;
    T w = valid ? T(1) : T(0);
    T Havg = T(0.5) * (Hm + Hp);
    T bm = M<T>::max(bedm, -rho_ratio<T>() * Hm), bp = M<T>::max(bedp, -rho_ratio<T>() * Hp);
    T dbm = bedm > -rho_ratio<T>() * Hm ? T(0) : -rho_ratio<T>();
    T dbp = bedp > -rho_ratio<T>() * Hp ? T(0) : -rho_ratio<T>();
    T dS = (bp + Hp) - (bm + Hm);
    o.res = Havg * dS * dxi * w;
    o.d_Hm = (T(0.5) * dS * dxi - Havg * (T(1) + dbm) * dxi) * w;
    o.d_Hp = (T(0.5) * dS * dxi + Havg * (T(1) + dbp) * dxi) * w;
    return o;
}

// Upwind face flux (flux.cu:39-64, :110-135).  For x-faces a = left cell,
// b = right cell, q = H_avg u - 0.5|u|(H_b - H_a).  For y-faces a = bottom
// (row i), b = top (row i-1), q = H_avg v - 0.5|v|(H_top - H_bottom).
template <typename T> struct Flux {
    T res, d_vel, d_Ha, d_Hb;
};
template <typename T> __device__ __forceinline__ Flux<T> upwind_flux(T vel, T Ha, T Hb, bool valid) {
    Flux<T> o;
    T w = valid ? T(1) : T(0);
    T Havg = T(0.5) * (Ha + Hb);
    T m = M<T>::abs(vel);
    T s = M<T>::copysign(T(1), vel);
    o.res = (Havg * vel - T(0.5) * m * (Hb - Ha)) * w;
    o.d_vel = (Havg - T(0.5) * s * (Hb - Ha)) * w;
    o.d_Ha = T(0.5) * (vel + m) * w;
    o.d_Hb = T(0.5) * (vel - m) * w;
    return o;
}

// Calving sink -c (1-g) H (flux.cu:187-211).
template <typename T> struct Calving {
    T res, d_H;
};
template <typename T> __device__ __forceinline__ Calving<T> calving_g(T H, T g, const Phys<T>& p) {
    Calving<T> o;
    o.res = -p.calving_rate * (T(1) - g) * H;
    o.d_H = -p.calving_rate * (T(1) - g);
    if (p.gl_deriv) o.d_H += p.calving_rate * H * (rho_ratio<T>() * (p.sig_c * g * (T(1) - g)));
    return o;
}
template <typename T> __device__ __forceinline__ Calving<T> calving(T H, T bed, const Phys<T>& p) {
    return calving_g(H, sigmoid(bed + rho_ratio<T>() * H, p.sig_c), p);
}

// Cell viscosity from its 4 faces and the 8 neighbouring faces of the 4
// corner shear rates (viscosity.cu:61-112); optional tangent (viscosity.cu:4-59).
template <typename T> struct EtaIn {
    T ul, ur, vt, vb;             // own faces
    T u_tl, u_tr, u_bl, u_br;     // u at (i-1,j), (i-1,j+1), (i+1,j), (i+1,j+1)
    T v_lt, v_rt, v_lb, v_rb;     // v at (i,j-1), (i,j+1), (i+1,j-1), (i+1,j+1)
};
template <typename T> struct EtaOut {
    T eta, eII, exy[4], ux, vy;
};
template <typename T>
__device__ __forceinline__ EtaOut<T> cell_eta(const EtaIn<T>& a, T Bc, int i, int j, int ny, int nx,
                                              const Phys<T>& p) {
    EtaOut<T> o;
    T dxi = p.dxi;
    o.ux = (a.ur - a.ul) * dxi;
    o.vy = (a.vt - a.vb) * dxi;
    T mtl = (i > 0 && j > 0) ? T(1) : T(0);
    T mtr = (i > 0 && j < nx - 1) ? T(1) : T(0);
    T mbl = (i < ny - 1 && j > 0) ? T(1) : T(0);
    T mbr = (i < ny - 1 && j < nx - 1) ? T(1) : T(0);
    o.exy[0] = T(0.5) * ((a.u_tl - a.ul) * dxi + (a.vt - a.v_lt) * dxi) * mtl;
    o.exy[1] = T(0.5) * ((a.u_tr - a.ur) * dxi + (a.v_rt - a.vt) * dxi) * mtr;
    o.exy[2] = T(0.5) * ((a.ul - a.u_bl) * dxi + (a.vb - a.v_lb) * dxi) * mbl;
    o.exy[3] = T(0.5) * ((a.ur - a.u_br) * dxi + (a.v_rb - a.vb) * dxi) * mbr;
    T e2 = T(0.25) * (o.exy[0] * o.exy[0] + o.exy[1] * o.exy[1] + o.exy[2] * o.exy[2] + o.exy[3] * o.exy[3]);
    o.eII = o.ux * o.ux + o.vy * o.vy + o.ux * o.vy + e2 + p.eps_reg;
    o.eta = T(0.5) * Bc * M<T>::pow(o.eII, p.glen_exp);
    return o;
}
// Tangent of eta for a tangent (du, dv) of the same 12 faces.
template <typename T>
__device__ __forceinline__ T cell_eta_tangent(const EtaOut<T>& e, const EtaIn<T>& d, T Bc, int i, int j, int ny,
                                              int nx, const Phys<T>& p) {
    T dxi = p.dxi;
    T dux = (d.ur - d.ul) * dxi;
    T dvy = (d.vt - d.vb) * dxi;
    T mtl = (i > 0 && j > 0) ? T(1) : T(0);
    T mtr = (i > 0 && j < nx - 1) ? T(1) : T(0);
    T mbl = (i < ny - 1 && j > 0) ? T(1) : T(0);
    T mbr = (i < ny - 1 && j < nx - 1) ? T(1) : T(0);
    T de0 = T(0.5) * ((d.u_tl - d.ul) * dxi + (d.vt - d.v_lt) * dxi) * mtl;
    T de1 = T(0.5) * ((d.u_tr - d.ur) * dxi + (d.v_rt - d.vt) * dxi) * mtr;
    T de2 = T(0.5) * ((d.ul - d.u_bl) * dxi + (d.vb - d.v_lb) * dxi) * mbl;
    T de3 = T(0.5) * ((d.ur - d.u_br) * dxi + (d.v_rb - d.vb) * dxi) * mbr;
    T de2sum = T(0.25) * (T(2) * e.exy[0] * de0 + T(2) * e.exy[1] * de1 + T(2) * e.exy[2] * de2 +
                          T(2) * e.exy[3] * de3);
    T deII = T(2) * e.ux * dux + T(2) * e.vy * dvy + (e.ux * dvy + e.vy * dux) + de2sum;
    return T(0.5) * Bc * (p.glen_exp * M<T>::pow(e.eII, p.glen_exp - T(1)) * deII);
}

// Load the 12 faces around cell (i,j) from a u/v pair (clamped).
template <typename T>
__device__ __forceinline__ EtaIn<T> eta_inputs(const T* __restrict__ u, const T* __restrict__ v, int i, int j,
                                               int ny, int nx) {
    EtaIn<T> a;
    a.ul = ldu(u, i, j, ny, nx);
    a.ur = ldu(u, i, j + 1, ny, nx);
    a.vt = ldv(v, i, j, ny, nx);
    a.vb = ldv(v, i + 1, j, ny, nx);
    a.u_tl = ldu(u, i - 1, j, ny, nx);
    a.u_tr = ldu(u, i - 1, j + 1, ny, nx);
    a.u_bl = ldu(u, i + 1, j, ny, nx);
    a.u_br = ldu(u, i + 1, j + 1, ny, nx);
    a.v_lt = ldv(v, i, j - 1, ny, nx);
    a.v_rt = ldv(v, i, j + 1, ny, nx);
    a.v_lb = ldv(v, i + 1, j - 1, ny, nx);
    a.v_rb = ldv(v, i + 1, j + 1, ny, nx);
    return a;
}

// Unpivoted Doolittle 5x5 solve, same elimination order as
// glide/cuda/common.cu:132-175.  A is overwritten.
template <typename T> __device__ __forceinline__ void lu5_solve(T (&A)[25], const T (&b)[5], T (&x)[5]) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
        T inv = T(1) / A[k * 5 + k];
#pragma unroll
        for (int i = k + 1; i < 5; i++) {
            A[i * 5 + k] *= inv;
#pragma unroll
            for (int j = k + 1; j < 5; j++) A[i * 5 + j] -= A[i * 5 + k] * A[k * 5 + j];
        }
    }
    T y[5];
    y[0] = b[0];
    y[1] = b[1] - A[5] * y[0];
    y[2] = b[2] - A[10] * y[0] - A[11] * y[1];
    y[3] = b[3] - A[15] * y[0] - A[16] * y[1] - A[17] * y[2];
    y[4] = b[4] - A[20] * y[0] - A[21] * y[1] - A[22] * y[2] - A[23] * y[3];
    x[4] = y[4] / A[24];
    x[3] = (y[3] - A[19] * x[4]) / A[18];
    x[2] = (y[2] - A[13] * x[3] - A[14] * x[4]) / A[12];
    x[1] = (y[1] - A[7] * x[2] - A[8] * x[3] - A[9] * x[4]) / A[6];
    x[0] = (y[0] - A[1] * x[1] - A[2] * x[2] - A[3] * x[3] - A[4] * x[4]) / A[0];
}

// error reporting from kernels: set a device flag, never trap
__device__ __forceinline__ void set_error(int* flag, int code) {
    if (flag) atomicCAS(flag, 0, code);
}

}  // namespace glide
