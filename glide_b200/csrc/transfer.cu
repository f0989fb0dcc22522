// Multigrid transfers (glide/cuda/utility.cu:1-337), the element-wise steps
// of the FASCD / adjoint V-cycles (glide/solver.py) fused into single passes,
// and deterministic FP64 reductions for the convergence norms.
#include "glide_common.cuh"

namespace glide {

constexpr int EW = 256;

static inline unsigned nblk(int64_t n) { return unsigned((n + EW - 1) / EW); }

// --------------------------------------------------------------------------
// restriction; sizes are given on the coarse grid (nyc, nxc), batch on grid.y
// --------------------------------------------------------------------------
template <typename T>
__global__ void restrict_u_k(const T* __restrict__ uf, T* __restrict__ uc, int nyc, int nxc, int64_t sf, int64_t sc) {
    const int64_t n = int64_t(nyc) * (nxc + 1);
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uf += blockIdx.y * sf; uc += blockIdx.y * sc;
    const int J = int(k / (nxc + 1)), I = int(k % (nxc + 1));
    const int W = 2 * nxc + 1;
    uc[k] = T(0.5) * (uf[int64_t(2 * J) * W + 2 * I] + uf[int64_t(2 * J + 1) * W + 2 * I]);
}
template <typename T>
__global__ void restrict_v_k(const T* __restrict__ vf, T* __restrict__ vc, int nyc, int nxc, int64_t sf, int64_t sc) {
    const int64_t n = int64_t(nyc + 1) * nxc;
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    vf += blockIdx.y * sf; vc += blockIdx.y * sc;
    const int J = int(k / nxc), I = int(k % nxc);
    const int W = 2 * nxc;
    vc[k] = T(0.5) * (vf[int64_t(2 * J) * W + 2 * I] + vf[int64_t(2 * J) * W + 2 * I + 1]);
}
template <typename T, bool MAX>
__global__ void restrict_c_k(const T* __restrict__ hf, T* __restrict__ hc, int nyc, int nxc, int64_t sf, int64_t sc) {
    const int64_t n = int64_t(nyc) * nxc;
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    hf += blockIdx.y * sf; hc += blockIdx.y * sc;
    const int J = int(k / nxc), I = int(k % nxc);
    const int W = 2 * nxc;
    const T a = hf[int64_t(2 * J) * W + 2 * I], b = hf[int64_t(2 * J) * W + 2 * I + 1];
    const T c = hf[int64_t(2 * J + 1) * W + 2 * I], d = hf[int64_t(2 * J + 1) * W + 2 * I + 1];
    hc[k] = MAX ? M<T>::max(M<T>::max(a, b), M<T>::max(c, d)) : T(0.25) * (a + b + c + d);
}

// --------------------------------------------------------------------------
// prolongation (utility.cu:21-54, 104-123, 145-178 linear/injection;
// 180-337 bilinear); mode 0: out = P(c), mode 1: out += P(c)
// --------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T bilinear(const T* __restrict__ c, int stride, T Jf, T If, int jmax, int imax) {
    Jf = M<T>::max(T(0), M<T>::min(Jf, T(jmax)));
    If = M<T>::max(T(0), M<T>::min(If, T(imax)));
    const int Jl = int(Jf), Il = int(If);
    const int Jh = min(Jl + 1, jmax), Ih = min(Il + 1, imax);
    const T ty = Jf - T(Jl), tx = If - T(Il);
    const T v00 = c[int64_t(Jl) * stride + Il], v01 = c[int64_t(Jl) * stride + Ih];
    const T v10 = c[int64_t(Jh) * stride + Il], v11 = c[int64_t(Jh) * stride + Ih];
    return (T(1) - ty) * ((T(1) - tx) * v00 + tx * v01) + ty * ((T(1) - tx) * v10 + tx * v11);
}

template <typename T>
__global__ void prolong_k(int field, int smooth, int mode, const T* __restrict__ c, T* __restrict__ out, int nyc,
                          int nxc, int64_t sc, int64_t sf) {
    const int nyf = 2 * nyc, nxf = 2 * nxc;
    const int rows = field == 1 ? nyf + 1 : nyf, cols = field == 0 ? nxf + 1 : nxf;
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= int64_t(rows) * cols) return;
    c += blockIdx.y * sc; out += blockIdx.y * sf;
    const int j = int(k / cols), i = int(k % cols);
    T val;
    if (field == 0) {
        if (smooth) {
            val = bilinear(c, nxc + 1, (T(j) - T(0.5)) * T(0.5), T(i) * T(0.5), nyc - 1, nxc);
        } else {
            const int64_t row = int64_t(j / 2) * (nxc + 1);
            const int I = i / 2;
            val = (i % 2 == 0) ? c[row + I] : (I < nxc ? T(0.5) * (c[row + I] + c[row + I + 1]) : c[row + I]);
        }
    } else if (field == 1) {
        if (smooth) {
            val = bilinear(c, nxc, T(j) * T(0.5), (T(i) - T(0.5)) * T(0.5), nyc, nxc - 1);
        } else {
            const int J = j / 2, I = i / 2;
            val = (j % 2 == 0) ? c[int64_t(J) * nxc + I]
                               : (J < nyc ? T(0.5) * (c[int64_t(J) * nxc + I] + c[int64_t(J + 1) * nxc + I])
                                          : c[int64_t(J) * nxc + I]);
        }
    } else {
        val = smooth ? bilinear(c, nxc, (T(j) - T(0.5)) * T(0.5), (T(i) - T(0.5)) * T(0.5), nyc - 1, nxc - 1)
                     : c[int64_t(j / 2) * nxc + i / 2];
    }
    if (mode == 0) out[k] = val;
    else out[k] += val;
}

// --------------------------------------------------------------------------
// fused element-wise V-cycle steps
// --------------------------------------------------------------------------
// out = a*x + b*y (y may be null)
template <typename T>
__global__ void lincomb_k(T* __restrict__ out, const T* __restrict__ x, T a, const T* __restrict__ y, T b, int64_t n) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    T v = a * x[k];
    if (y) v += b * y[k];
    out[k] = v;
}
template <typename T> __global__ void fill_k(T* __restrict__ out, T val, int64_t n) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) out[k] = val;
}
// mask = H <= gamma + tol (glide/grid.py:332-334)
template <typename T>
__global__ void mask_le_k(T* __restrict__ mask, const T* __restrict__ H, const T* __restrict__ gamma, T tol, int64_t n) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) mask[k] = H[k] <= gamma[k] + tol ? T(1) : T(0);
}
// Constraint restriction of the FASCD pre-smoothing step
// (glide/solver.py:101-108): chi_c = maxpool(chi_f),
// gamma_f = w_H + (inject(-chi_c) + chi_f).
template <typename T>
__global__ void constraint_down_k(T* __restrict__ chi_c, T* __restrict__ gamma_f, const T* __restrict__ chi_f,
                                  const T* __restrict__ wH_f, int nyc, int nxc, int64_t sf, int64_t sc) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= int64_t(nyc) * nxc) return;
    chi_f += blockIdx.y * sf; wH_f += blockIdx.y * sf; gamma_f += blockIdx.y * sf; chi_c += blockIdx.y * sc;
    const int J = int(k / nxc), I = int(k % nxc);
    const int W = 2 * nxc;
    const int64_t f00 = int64_t(2 * J) * W + 2 * I, f01 = f00 + 1, f10 = f00 + W, f11 = f10 + 1;
    const T a = chi_f[f00], b = chi_f[f01], c = chi_f[f10], d = chi_f[f11];
    const T m = M<T>::max(M<T>::max(a, b), M<T>::max(c, d));
    chi_c[k] = m;
    gamma_f[f00] = wH_f[f00] + (-m + a);
    gamma_f[f01] = wH_f[f01] + (-m + b);
    gamma_f[f10] = wH_f[f10] + (-m + c);
    gamma_f[f11] = wH_f[f11] + (-m + d);
}

// --------------------------------------------------------------------------
// deterministic reductions: per-block partial sums (FP64) then one block
// sums the partials in a fixed order.
// parts[3*b + {0,1,2}] = sum r_u^2, sum r_v^2, sum FB(r_H, H-gamma)^2
// --------------------------------------------------------------------------
constexpr int RB = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < RB / 32; k++) s += sh[k];
    }
    __syncthreads();
    return s;
}

template <typename T>
__global__ void __launch_bounds__(RB) norms_partial_k(double* __restrict__ parts, const T* __restrict__ r_u,
                                                      const T* __restrict__ r_v, const T* __restrict__ r_H,
                                                      const T* __restrict__ H, const T* __restrict__ gamma,
                                                      int64_t nu, int64_t nv, int64_t nc) {
    __shared__ double sh[RB / 32];
    double su = 0, sv = 0, sh_ = 0;
    const int64_t stride = int64_t(gridDim.x) * RB;
    for (int64_t k = int64_t(blockIdx.x) * RB + threadIdx.x; k < nu; k += stride) {
        double x = double(r_u[k]);
        su += x * x;
    }
    for (int64_t k = int64_t(blockIdx.x) * RB + threadIdx.x; k < nv; k += stride) {
        double x = double(r_v[k]);
        sv += x * x;
    }
    for (int64_t k = int64_t(blockIdx.x) * RB + threadIdx.x; k < nc; k += stride) {
        T a = r_H[k], b = H[k] - gamma[k];
        double fb = double(a + b - M<T>::sqrt(a * a + b * b));
        sh_ += fb * fb;
    }
    double t0 = block_sum(su, sh);
    double t1 = block_sum(sv, sh);
    double t2 = block_sum(sh_, sh);
    if (threadIdx.x == 0) {
        parts[3 * blockIdx.x + 0] = t0;
        parts[3 * blockIdx.x + 1] = t1;
        parts[3 * blockIdx.x + 2] = t2;
    }
}
// Sum of the per-block partials in a fixed order (thread t adds parts t, t+RB,
// ... in sequence, then a fixed shuffle/shared-memory tree): deterministic.
__global__ void __launch_bounds__(RB) norms_final_k(double* __restrict__ out, const double* __restrict__ parts,
                                                     int nparts) {
    __shared__ double sh[RB / 32];
    double a = 0, b = 0, c = 0;
    for (int k = threadIdx.x; k < nparts; k += RB) {
        a += parts[3 * k];
        b += parts[3 * k + 1];
        c += parts[3 * k + 2];
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    c = block_sum(c, sh);
    if (threadIdx.x == 0) {
        out[0] = a;
        out[1] = b;
        out[2] = c;
    }
}

// Coarse-correction line search (finest level): pick the candidate step with
// the smallest residual norm.  norms holds 3 sums of squares per candidate.
__global__ void ls_pick_k(double* __restrict__ alpha_out, const double* __restrict__ norms, int k) {
    const double alphas[4] = {1.0, 0.5, 0.25, 0.0};  // GLIDE_LS_CANDIDATES, best first on ties
    if (threadIdx.x != 0 || blockIdx.x != 0 || k < 1 || k > 4) return;
    int best = 0;
    double bn = norms[0] + norms[1] + norms[2];
    for (int j = 1; j < k; j++) {
        const double nj = norms[3 * j] + norms[3 * j + 1] + norms[3 * j + 2];
        if (nj < bn) {  // NaN candidates never win
            bn = nj;
            best = j;
        }
    }
    alpha_out[0] = alphas[best];
}

// out = x + alpha[0] * y with alpha read on the device.
template <typename T>
__global__ void axpy_dev_k(T* __restrict__ out, const T* __restrict__ x, const double* __restrict__ alpha,
                           const T* __restrict__ y, int64_t n) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out[k] = x[k] + T(alpha[0]) * y[k];
}


// --------------------------------------------------------------------------
// launchers (batch count nb on grid.y)
// --------------------------------------------------------------------------
template <typename T>
int launch_restrict(int field, int use_max, const void* fine, void* coarse, int nyc, int nxc, int nb,
                    cudaStream_t s) {
    const int nyf = 2 * nyc, nxf = 2 * nxc;
    if (field == 0) {
        glide::count_launch(), restrict_u_k<T><<<dim3(nblk(int64_t(nyc) * (nxc + 1)), nb), EW, 0, s>>>(
            (const T*)fine, (T*)coarse, nyc, nxc, int64_t(nyf) * (nxf + 1), int64_t(nyc) * (nxc + 1));
    } else if (field == 1) {
        glide::count_launch(), restrict_v_k<T><<<dim3(nblk(int64_t(nyc + 1) * nxc), nb), EW, 0, s>>>(
            (const T*)fine, (T*)coarse, nyc, nxc, int64_t(nyf + 1) * nxf, int64_t(nyc + 1) * nxc);
    } else if (use_max) {
        glide::count_launch(), restrict_c_k<T, true><<<dim3(nblk(int64_t(nyc) * nxc), nb), EW, 0, s>>>(
            (const T*)fine, (T*)coarse, nyc, nxc, int64_t(nyf) * nxf, int64_t(nyc) * nxc);
    } else {
        glide::count_launch(), restrict_c_k<T, false><<<dim3(nblk(int64_t(nyc) * nxc), nb), EW, 0, s>>>(
            (const T*)fine, (T*)coarse, nyc, nxc, int64_t(nyf) * nxf, int64_t(nyc) * nxc);
    }
    return (int)cudaGetLastError();
}

template <typename T>
int launch_prolong(int field, int smooth, int add, const void* coarse, void* fine, int nyc, int nxc, int nb,
                   cudaStream_t s) {
    const int nyf = 2 * nyc, nxf = 2 * nxc;
    int64_t nf = field == 0 ? int64_t(nyf) * (nxf + 1) : field == 1 ? int64_t(nyf + 1) * nxf : int64_t(nyf) * nxf;
    int64_t ncs = field == 0 ? int64_t(nyc) * (nxc + 1) : field == 1 ? int64_t(nyc + 1) * nxc : int64_t(nyc) * nxc;
    glide::count_launch(), prolong_k<T><<<dim3(nblk(nf), nb), EW, 0, s>>>(field, smooth, add, (const T*)coarse, (T*)fine, nyc, nxc, ncs, nf);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_lincomb(void* out, const void* x, double a, const void* y, double b, int64_t n, cudaStream_t s) {
    if (n <= 0) return 0;
    glide::count_launch(), lincomb_k<T><<<nblk(n), EW, 0, s>>>((T*)out, (const T*)x, T(a), (const T*)y, T(b), n);
    return (int)cudaGetLastError();
}
template <typename T> int launch_fill(void* out, double val, int64_t n, cudaStream_t s) {
    if (n <= 0) return 0;
    glide::count_launch(), fill_k<T><<<nblk(n), EW, 0, s>>>((T*)out, T(val), n);
    return (int)cudaGetLastError();
}
template <typename T>
int launch_mask_le(void* mask, const void* H, const void* gamma, double tol, int64_t n, cudaStream_t s) {
    if (n <= 0) return 0;
    glide::count_launch(), mask_le_k<T><<<nblk(n), EW, 0, s>>>((T*)mask, (const T*)H, (const T*)gamma, T(tol), n);
    return (int)cudaGetLastError();
}
template <typename T>
int launch_constraint_down(void* chi_c, void* gamma_f, const void* chi_f, const void* wH_f, int nyc, int nxc, int nb,
                           cudaStream_t s) {
    glide::count_launch(), constraint_down_k<T><<<dim3(nblk(int64_t(nyc) * nxc), nb), EW, 0, s>>>(
        (T*)chi_c, (T*)gamma_f, (const T*)chi_f, (const T*)wH_f, nyc, nxc, int64_t(4) * nyc * nxc,
        int64_t(nyc) * nxc);
    return (int)cudaGetLastError();
}

int norms_parts_count(int64_t n) {
    int64_t b = (n + RB - 1) / RB;
    if (b > 1184) b = 1184;  // 8 CTAs per SM on 148 SMs
    if (b < 1) b = 1;
    return int(b);
}

template <typename T>
int launch_norms(double* out3, double* parts, const void* r_u, const void* r_v, const void* r_H, const void* H,
                 const void* gamma, int64_t nu, int64_t nv, int64_t nc, cudaStream_t s) {
    const int nb = norms_parts_count(nu > nc ? nu : nc);
    glide::count_launch(), norms_partial_k<T><<<nb, RB, 0, s>>>(parts, (const T*)r_u, (const T*)r_v, (const T*)r_H, (const T*)H,
                                         (const T*)gamma, nu, nv, nc);
    glide::count_launch(), norms_final_k<<<1, RB, 0, s>>>(out3, parts, nb);
    return (int)cudaGetLastError();
}

int launch_ls_pick(double* alpha_out, const double* norms, int k, cudaStream_t s) {
    glide::count_launch(), ls_pick_k<<<1, 32, 0, s>>>(alpha_out, norms, k);
    return (int)cudaGetLastError();
}

template <typename T>
int launch_axpy_dev(void* out, const void* x, const double* alpha, const void* y, int64_t n, cudaStream_t s) {
    glide::count_launch(), axpy_dev_k<T><<<nblk(n), EW, 0, s>>>((T*)out, (const T*)x, alpha, (const T*)y, n);
    return (int)cudaGetLastError();
}

#define INST(T)                                                                                                   \
    template int launch_restrict<T>(int, int, const void*, void*, int, int, int, cudaStream_t);                    \
    template int launch_prolong<T>(int, int, int, const void*, void*, int, int, int, cudaStream_t);                \
    template int launch_lincomb<T>(void*, const void*, double, const void*, double, int64_t, cudaStream_t);        \
    template int launch_fill<T>(void*, double, int64_t, cudaStream_t);                                             \
    template int launch_mask_le<T>(void*, const void*, const void*, double, int64_t, cudaStream_t);                \
    template int launch_constraint_down<T>(void*, void*, const void*, const void*, int, int, int, cudaStream_t);   \
    template int launch_norms<T>(double*, double*, const void*, const void*, const void*, const void*, const void*, \
                                 int64_t, int64_t, int64_t, cudaStream_t);                                         \
    template int launch_axpy_dev<T>(void*, const void*, const double*, const void*, int64_t, cudaStream_t);
INST(float)
INST(double)
#undef INST

}  // namespace glide
