// Fused loss kernels for the inverse problem (glide/physics.py:262-411): one
// pass computes a misfit and its gradient, one pass the Tikhonov term and its
// gradient; the loss is summed in FP64 per block and the block sums are added
// in a fixed order, so results are deterministic.
//
// Misfit, per component c in {u, v} with d = c - c_obs and NaN differences
// set to 0 (glide/physics.py:276-283):
//   kind 0 (abs):   L_c = mean |d|,               dL/dc = sign(d) / n_u
//   kind 1 (huber): L_c = mean sqrt(d^2 + eps),   dL/dc = d / sqrt(d^2 + eps) / n_u
// L = L_u + L_v.  Both gradients divide by the number of u entries, as the
// reference's gradient helpers do (glide/physics.py:318-320).
// Tikhonov (glide/physics.py:382-411): L = 1/2 sum of squared differences of
// horizontal and vertical neighbours; grad = sum over in-domain neighbours of
// (f_c - f_nb).
#include "glide_common.cuh"

namespace glide {

constexpr int LB = 256;

__device__ __forceinline__ double block_sum_loss(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < LB / 32; k++) s += sh[k];
    }
    __syncthreads();
    return s;
}

template <typename T>
__device__ __forceinline__ double misfit_term(T c, T obs, int kind, T eps, T inv_n, T& grad) {
    T d = c - obs;
    if (isnan(d)) d = T(0);
    if (kind == 0) {
        grad = (d > T(0) ? T(1) : (d < T(0) ? T(-1) : T(0))) * inv_n;
        return fabs(double(d));
    }
    const T s = M<T>::sqrt(d * d + eps);
    grad = d / s * inv_n;
    return double(s);
}

template <typename T>
__global__ void __launch_bounds__(LB) misfit_partial_k(double* __restrict__ parts, T* __restrict__ grad_u,
                                                       T* __restrict__ grad_v, const T* __restrict__ u,
                                                       const T* __restrict__ v, const T* __restrict__ u_obs,
                                                       const T* __restrict__ v_obs, int64_t nu, int64_t nv,
                                                       int kind, T eps, T inv_n) {
    __shared__ double sh[LB / 32];
    double su = 0, sv = 0;
    const int64_t stride = int64_t(gridDim.x) * LB;
    for (int64_t k = int64_t(blockIdx.x) * LB + threadIdx.x; k < nu; k += stride) {
        T g;
        su += misfit_term(u[k], u_obs[k], kind, eps, inv_n, g);
        grad_u[k] = g;
    }
    for (int64_t k = int64_t(blockIdx.x) * LB + threadIdx.x; k < nv; k += stride) {
        T g;
        sv += misfit_term(v[k], v_obs[k], kind, eps, inv_n, g);
        grad_v[k] = g;
    }
    const double tu = block_sum_loss(su, sh);
    const double tv = block_sum_loss(sv, sh);
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = tu;
        parts[2 * blockIdx.x + 1] = tv;
    }
}

// out[0] = sum_u / nu + sum_v / nv, out[1] = sum_u, out[2] = sum_v
__global__ void __launch_bounds__(LB) misfit_final_k(double* __restrict__ out, const double* __restrict__ parts,
                                                     int nparts, double nu, double nv) {
    __shared__ double sh[LB / 32];
    double a = 0, b = 0;
    for (int k = threadIdx.x; k < nparts; k += LB) {
        a += parts[2 * k];
        b += parts[2 * k + 1];
    }
    a = block_sum_loss(a, sh);
    b = block_sum_loss(b, sh);
    if (threadIdx.x == 0) {
        out[0] = a / nu + b / nv;
        out[1] = a;
        out[2] = b;
    }
}

template <typename T>
__global__ void __launch_bounds__(LB) tikhonov_partial_k(double* __restrict__ parts, T* __restrict__ grad,
                                                         const T* __restrict__ f, int ny, int nx) {
    __shared__ double sh[LB / 32];
    double s = 0;
    const int64_t n = int64_t(ny) * nx;
    const int64_t stride = int64_t(gridDim.x) * LB;
    for (int64_t k = int64_t(blockIdx.x) * LB + threadIdx.x; k < n; k += stride) {
        const int i = int(k / nx), j = int(k - int64_t(i) * nx);
        const T c = f[k];
        T g = T(0);
        if (j + 1 < nx) {
            const T d = f[k + 1] - c;
            s += 0.5 * double(d) * double(d);
            g -= d;
        }
        if (i + 1 < ny) {
            const T d = f[k + nx] - c;
            s += 0.5 * double(d) * double(d);
            g -= d;
        }
        if (j > 0) g += c - f[k - 1];
        if (i > 0) g += c - f[k - nx];
        grad[k] = g;
    }
    const double t = block_sum_loss(s, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = t;
}

__global__ void __launch_bounds__(LB) sum_final_k(double* __restrict__ out, const double* __restrict__ parts,
                                                  int nparts) {
    __shared__ double sh[LB / 32];
    double a = 0;
    for (int k = threadIdx.x; k < nparts; k += LB) a += parts[k];
    a = block_sum_loss(a, sh);
    if (threadIdx.x == 0) out[0] = a;
}

int loss_parts_count(int64_t n) {
    int64_t b = (n + LB - 1) / LB;
    if (b > 1184) b = 1184;  // 8 CTAs per SM on 148 SMs
    if (b < 1) b = 1;
    return int(b);
}

template <typename T>
int launch_misfit(int kind, double eps, const void* u, const void* v, const void* u_obs, const void* v_obs,
                  int64_t nu, int64_t nv, void* grad_u, void* grad_v, double* out, double* parts, cudaStream_t s) {
    const int nb = loss_parts_count(nu > nv ? nu : nv);
    glide::count_launch(), misfit_partial_k<T><<<nb, LB, 0, s>>>(parts, (T*)grad_u, (T*)grad_v, (const T*)u,
                                                                 (const T*)v, (const T*)u_obs, (const T*)v_obs, nu,
                                                                 nv, kind, T(eps), T(1.0 / double(nu)));
    glide::count_launch(), misfit_final_k<<<1, LB, 0, s>>>(out, parts, nb, double(nu), double(nv));
    return (int)cudaGetLastError();
}

template <typename T>
int launch_tikhonov(const void* f, int ny, int nx, void* grad, double* out, double* parts, cudaStream_t s) {
    const int nb = loss_parts_count(int64_t(ny) * nx);
    glide::count_launch(), tikhonov_partial_k<T><<<nb, LB, 0, s>>>(parts, (T*)grad, (const T*)f, ny, nx);
    glide::count_launch(), sum_final_k<<<1, LB, 0, s>>>(out, parts, nb);
    return (int)cudaGetLastError();
}

}  // namespace glide

using namespace glide;

extern "C" int glide_loss_parts(int64_t n) { return 2 * loss_parts_count(n); }

extern "C" int glide_misfit(int dtype, int kind, double eps, const void* u, const void* v, const void* u_obs,
                            const void* v_obs, int64_t nu, int64_t nv, void* grad_u, void* grad_v, double* out3,
                            double* parts, void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (kind != 0 && kind != 1) return GLIDE_E_SHAPE;
    if (nu < 1 || nv < 1) return GLIDE_E_SHAPE;
    if (!u || !v || !u_obs || !v_obs || !grad_u || !grad_v || !out3 || !parts) return GLIDE_E_NULL;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == GLIDE_F32
               ? launch_misfit<float>(kind, eps, u, v, u_obs, v_obs, nu, nv, grad_u, grad_v, out3, parts, s)
               : launch_misfit<double>(kind, eps, u, v, u_obs, v_obs, nu, nv, grad_u, grad_v, out3, parts, s);
}

extern "C" int glide_tikhonov(int dtype, const void* field, int ny, int nx, void* grad, double* out1,
                              double* parts, void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (ny < 1 || nx < 1) return GLIDE_E_SHAPE;
    if (!field || !grad || !out1 || !parts) return GLIDE_E_NULL;
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == GLIDE_F32 ? launch_tikhonov<float>(field, ny, nx, grad, out1, parts, s)
                              : launch_tikhonov<double>(field, ny, nx, grad, out1, parts, s);
}
