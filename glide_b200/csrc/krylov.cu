// Vector kernels of the Newton-Krylov finishing solver and of the Anderson
// step (no counterpart in the reference, whose solver is a fixed number of
// FAS V-cycles): several dot products against one vector in one pass with
// FP64 accumulation (deterministic: per-block partials summed in a fixed
// order), linear combinations of stored vectors with device coefficients,
// and the element-wise steps of a Newton update in mixed precision.
#include "glide_common.cuh"

namespace glide {

constexpr int KB = 256;          // threads per block
constexpr int DOT_KMAX = 32;     // vectors per multi-dot / combine call
constexpr int DOT_MAX_BLOCKS = 1184;   // 8 blocks per SM on 148 SMs

int dots_parts_count(int64_t n) {
    int64_t b = (n + KB - 1) / KB;
    if (b > DOT_MAX_BLOCKS) b = DOT_MAX_BLOCKS;
    if (b < 1) b = 1;
    return int(b);
}

// parts[blk * K + i] = sum over this block's elements of V[i][j] * w[j]
// (FP64 products and sums); w is read once for all K vectors.
template <typename T, int K>
__global__ void __launch_bounds__(KB) multidot_partial_k(double* __restrict__ parts, const T* __restrict__ V,
                                                         int64_t ldv, const T* __restrict__ w, int64_t n, int k) {
    __shared__ double sh[KB / 32][K];
    double acc[K];
#pragma unroll
    for (int i = 0; i < K; i++) acc[i] = 0.0;
    const int64_t stride = int64_t(gridDim.x) * KB;
    for (int64_t j = int64_t(blockIdx.x) * KB + threadIdx.x; j < n; j += stride) {
        const double wj = double(w[j]);
#pragma unroll
        for (int i = 0; i < K; i++)
            if (i < k) acc[i] += double(V[int64_t(i) * ldv + j]) * wj;
    }
    const int wid = threadIdx.x / 32, lane = threadIdx.x % 32;
#pragma unroll
    for (int i = 0; i < K; i++) {
        if (i >= k) break;
        double v = acc[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[wid][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double s = 0.0;
        for (int q = 0; q < KB / 32; q++) s += sh[q][threadIdx.x];
        parts[int64_t(blockIdx.x) * k + threadIdx.x] = s;
    }
}

// out[i] = sum over blocks of parts[b * k + i], block i of the grid, fixed order.
__global__ void __launch_bounds__(KB) multidot_final_k(double* __restrict__ out, const double* __restrict__ parts,
                                                       int nparts, int k) {
    __shared__ double sh[KB / 32];
    const int i = blockIdx.x;
    double a = 0.0;
    for (int b = threadIdx.x; b < nparts; b += KB) a += parts[int64_t(b) * k + i];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (threadIdx.x % 32 == 0) sh[threadIdx.x / 32] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < KB / 32; q++) s += sh[q];
        out[i] = s;
    }
}

// out[j] = beta * out[j] + alpha * sum_i coef[i] * V[i][j]  (beta = 0: out is not read)
template <typename T>
__global__ void __launch_bounds__(KB) combine_k(T* __restrict__ out, const T* __restrict__ V, int64_t ldv,
                                                const double* __restrict__ coef, double alpha, double beta,
                                                int64_t n, int k) {
    __shared__ T c[DOT_KMAX];
    if (threadIdx.x < k) c[threadIdx.x] = T(alpha * coef[threadIdx.x]);
    __syncthreads();
    const int64_t stride = int64_t(gridDim.x) * KB;
    for (int64_t j = int64_t(blockIdx.x) * KB + threadIdx.x; j < n; j += stride) {
        T s = beta == 0.0 ? T(0) : T(beta) * out[j];
        for (int i = 0; i < k; i++) s += c[i] * V[int64_t(i) * ldv + j];
        out[j] = s;
    }
}

// Right-hand side of one Newton step.  r is the FP64 residual F(U) - f of
// the state (faces first, then cells); a cell is in the active set when
// H - dt r_H <= gamma (the Vanka smoother's rule), and its row becomes the
// constraint H - gamma.  rhs = masked r, rraw = r and mask = the active set,
// all in the linear solver's precision TO (FP32 for the mixed path, FP64 for
// the FP64 path).
template <typename TO>
__global__ void newton_rhs_k(TO* __restrict__ rhs, TO* __restrict__ rraw, TO* __restrict__ mask,
                             const double* __restrict__ r, const double* __restrict__ H,
                             const double* __restrict__ gamma, double dt, int64_t n_faces, int64_t n_cells) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n_faces) {
        const TO x = TO(r[k]);
        rhs[k] = x;
        rraw[k] = x;
    } else if (k < n_faces + n_cells) {
        const int64_t c = k - n_faces;
        const double rH = r[k];
        const bool act = H[c] - dt * rH <= gamma[c];
        mask[c] = act ? TO(1) : TO(0);
        rhs[k] = TO(act ? H[c] - gamma[c] : rH);
        rraw[k] = TO(rH);
    }
}

// mask = (H - dt r_H <= gamma), cells of one level.
template <typename T>
__global__ void active_mask_k(T* __restrict__ mask, const T* __restrict__ H, const T* __restrict__ r_H,
                              const T* __restrict__ gamma, T dt, int64_t n) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < n) mask[k] = H[k] - dt * r_H[k] <= gamma[k] ? T(1) : T(0);
}

// U = base + alpha * d with H kept >= gamma (FP64 state; d in the linear
// solver's precision TD).
template <typename TD>
__global__ void newton_update_k(double* __restrict__ U, const double* __restrict__ base, const TD* __restrict__ d,
                                double alpha, const double* __restrict__ gamma, int64_t n_faces, int64_t n_cells) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n_faces + n_cells) return;
    double x = base[k] + alpha * double(d[k]);
    if (k >= n_faces) x = fmax(x, gamma[k - n_faces]);
    U[k] = x;
}

static inline unsigned nblocks(int64_t n) { return unsigned((n + KB - 1) / KB); }

// At most 16 vectors per pass (16 FP64 accumulators keep the kernel near 80
// registers and the SM full of warps); more vectors take a second pass.
template <typename T>
int launch_dots(int64_t n, int k, const void* V, int64_t ldv, const void* w, double* out, double* parts,
                cudaStream_t s) {
    const int nb = dots_parts_count(n);
    for (int i0 = 0; i0 < k; i0 += 16) {
        const int kk = k - i0 < 16 ? k - i0 : 16;
        const T* Vi = (const T*)V + int64_t(i0) * ldv;
        if (kk <= 8)
            glide::count_launch(), multidot_partial_k<T, 8><<<nb, KB, 0, s>>>(parts, Vi, ldv, (const T*)w, n, kk);
        else
            glide::count_launch(), multidot_partial_k<T, 16><<<nb, KB, 0, s>>>(parts, Vi, ldv, (const T*)w, n, kk);
        glide::count_launch(), multidot_final_k<<<kk, KB, 0, s>>>(out + i0, parts, nb, kk);
    }
    return (int)cudaGetLastError();
}

template <typename T>
int launch_combine(int64_t n, int k, const void* V, int64_t ldv, const double* coef, double alpha, void* out,
                   double beta, cudaStream_t s) {
    unsigned nb = nblocks(n);
    if (nb > unsigned(DOT_MAX_BLOCKS)) nb = DOT_MAX_BLOCKS;
    glide::count_launch(), combine_k<T><<<nb, KB, 0, s>>>((T*)out, (const T*)V, ldv, coef, alpha, beta, n, k);
    return (int)cudaGetLastError();
}

}  // namespace glide

using namespace glide;

extern "C" {

int glide_dots_parts(int64_t n) { return dots_parts_count(n); }

int glide_dots(int dtype, int64_t n, int k, const void* V, int64_t ldv, const void* w, double* out, double* parts,
               void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!V || !w || !out || !parts) return GLIDE_E_NULL;
    if (n < 1 || k < 1 || k > DOT_KMAX || ldv < n) return GLIDE_E_SHAPE;
    return dtype == GLIDE_F32 ? launch_dots<float>(n, k, V, ldv, w, out, parts, (cudaStream_t)stream)
                              : launch_dots<double>(n, k, V, ldv, w, out, parts, (cudaStream_t)stream);
}

int glide_combine(int dtype, int64_t n, int k, const void* V, int64_t ldv, const double* coef, double alpha,
                  void* out, double beta, void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!V || !coef || !out) return GLIDE_E_NULL;
    if (n < 1 || k < 1 || k > DOT_KMAX || ldv < n) return GLIDE_E_SHAPE;
    return dtype == GLIDE_F32 ? launch_combine<float>(n, k, V, ldv, coef, alpha, out, beta, (cudaStream_t)stream)
                              : launch_combine<double>(n, k, V, ldv, coef, alpha, out, beta, (cudaStream_t)stream);
}

int glide_newton_rhs(const GlideLevelArgs* a64, const void* r64, void* rhs, void* rraw, void* mask, int lin_dtype,
                     void* stream) {
    if (!a64 || !r64 || !rhs || !rraw || !mask || !a64->H || !a64->gamma) return GLIDE_E_NULL;
    if (a64->dtype != GLIDE_F64 || (lin_dtype != GLIDE_F32 && lin_dtype != GLIDE_F64)) return GLIDE_E_DTYPE;
    const int64_t nb = a64->nb, ny = a64->ny, nx = a64->nx;
    const int64_t nf = nb * (ny * (nx + 1) + (ny + 1) * nx), nc = nb * ny * nx;
    glide::count_launch();
    if (lin_dtype == GLIDE_F32)
        newton_rhs_k<float><<<nblocks(nf + nc), KB, 0, (cudaStream_t)stream>>>(
            (float*)rhs, (float*)rraw, (float*)mask, (const double*)r64, (const double*)a64->H,
            (const double*)a64->gamma, a64->dt, nf, nc);
    else
        newton_rhs_k<double><<<nblocks(nf + nc), KB, 0, (cudaStream_t)stream>>>(
            (double*)rhs, (double*)rraw, (double*)mask, (const double*)r64, (const double*)a64->H,
            (const double*)a64->gamma, a64->dt, nf, nc);
    return (int)cudaGetLastError();
}

int glide_active_mask(const GlideLevelArgs* a, const void* r_H, void* mask, void* stream) {
    if (!a || !r_H || !mask || !a->H || !a->gamma) return GLIDE_E_NULL;
    const int64_t n = int64_t(a->nb) * a->ny * a->nx;
    glide::count_launch();
    if (a->dtype == GLIDE_F32)
        active_mask_k<float><<<nblocks(n), KB, 0, (cudaStream_t)stream>>>(
            (float*)mask, (const float*)a->H, (const float*)r_H, (const float*)a->gamma, float(a->dt), n);
    else if (a->dtype == GLIDE_F64)
        active_mask_k<double><<<nblocks(n), KB, 0, (cudaStream_t)stream>>>(
            (double*)mask, (const double*)a->H, (const double*)r_H, (const double*)a->gamma, a->dt, n);
    else
        return GLIDE_E_DTYPE;
    return (int)cudaGetLastError();
}

int glide_newton_update(const GlideLevelArgs* a64, void* U64, const void* base64, const void* d, int d_dtype,
                        double alpha, void* stream) {
    if (!a64 || !U64 || !base64 || !d || !a64->gamma) return GLIDE_E_NULL;
    if (a64->dtype != GLIDE_F64 || (d_dtype != GLIDE_F32 && d_dtype != GLIDE_F64)) return GLIDE_E_DTYPE;
    const int64_t nb = a64->nb, ny = a64->ny, nx = a64->nx;
    const int64_t nf = nb * (ny * (nx + 1) + (ny + 1) * nx), nc = nb * ny * nx;
    glide::count_launch();
    if (d_dtype == GLIDE_F32)
        newton_update_k<float><<<nblocks(nf + nc), KB, 0, (cudaStream_t)stream>>>(
            (double*)U64, (const double*)base64, (const float*)d, alpha, (const double*)a64->gamma, nf, nc);
    else
        newton_update_k<double><<<nblocks(nf + nc), KB, 0, (cudaStream_t)stream>>>(
            (double*)U64, (const double*)base64, (const double*)d, alpha, (const double*)a64->gamma, nf, nc);
    return (int)cudaGetLastError();
}

}  // extern "C"
