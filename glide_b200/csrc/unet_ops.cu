// Data-movement kernels around the tensor-core GEMM for the learned guess:
// im2col of a 3x3 "same" convolution, its transpose (col2im, gather form so
// every output has one writer), BF16 transposes, and the pack/unpack between
// the solver's staggered fields and the network's NHWC tensors.
#include <cuda_bf16.h>
#include <stdint.h>

#include "glide_b200.h"

namespace glide {
void count_launch();
}

namespace glide {

// col[p, (ky*3+kx)*C + c] = x[b, y+ky-1, x+kx-1, c] (zero outside); p = (b*H + y)*W + x.
// Columns [9C, Kp) are zero.
__global__ void im2col3_k(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ col, int Bn, int H, int W,
                          int C, int Kp) {
    const int64_t total = int64_t(Bn) * H * W * Kp;
    for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const int k = int(idx % Kp);
        const int64_t p = idx / Kp;
        __nv_bfloat16 v = __float2bfloat16(0.0f);
        if (k < 9 * C) {
            const int tap = k / C, c = k % C;
            const int ky = tap / 3, kx = tap % 3;
            const int xx = int(p % W), yy = int((p / W) % H), b = int(p / (int64_t(W) * H));
            const int sy = yy + ky - 1, sx = xx + kx - 1;
            if (sy >= 0 && sy < H && sx >= 0 && sx < W) v = x[((int64_t(b) * H + sy) * W + sx) * C + c];
        }
        col[idx] = v;
    }
}

// dx[b,y,x,c] = sum_{ky,kx} dcol[p(b, y-ky+1, x-kx+1), (ky*3+kx)*C + c]
__global__ void col2im3_k(const float* __restrict__ dcol, float* __restrict__ dx, int Bn, int H, int W, int C, int Kp) {
    const int64_t total = int64_t(Bn) * H * W * C;
    for (int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; idx < total;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const int c = int(idx % C);
        const int64_t pix = idx / C;
        const int xx = int(pix % W), yy = int((pix / W) % H), b = int(pix / (int64_t(W) * H));
        float acc = 0.0f;
#pragma unroll
        for (int ky = 0; ky < 3; ky++) {
#pragma unroll
            for (int kx = 0; kx < 3; kx++) {
                const int oy = yy - ky + 1, ox = xx - kx + 1;
                if (oy >= 0 && oy < H && ox >= 0 && ox < W) {
                    const int64_t p = (int64_t(b) * H + oy) * W + ox;
                    acc += dcol[p * Kp + (ky * 3 + kx) * C + c];
                }
            }
        }
        dx[idx] = acc;
    }
}

// dst[c, r] = src[r, c]  (R x Cc -> Cc x R), BF16, 32x32 smem tiles
__global__ void transpose_bf16_k(const __nv_bfloat16* __restrict__ src, __nv_bfloat16* __restrict__ dst, int R,
                                 int Cc) {
    __shared__ __nv_bfloat16 t[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        t[k][threadIdx.x] = (r < R && c < Cc) ? src[int64_t(r) * Cc + c] : __float2bfloat16(0.0f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < Cc && r < R) dst[int64_t(c) * R + r] = t[threadIdx.x][k];
    }
}

static inline unsigned blocks_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return unsigned(b > 148 * 64 ? 148 * 64 : (b < 1 ? 1 : b));
}

}  // namespace glide

extern "C" int glide_im2col3_bf16(const void* x, void* col, int Bn, int H, int W, int C, int Kp, void* stream) {
    if (!x || !col) return GLIDE_E_NULL;
    if (Bn < 1 || H < 1 || W < 1 || C < 1 || Kp < 9 * C) return GLIDE_E_SHAPE;
    glide::count_launch(), glide::im2col3_k<<<glide::blocks_for(int64_t(Bn) * H * W * Kp), 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)x, (__nv_bfloat16*)col, Bn, H, W, C, Kp);
    return (int)cudaGetLastError();
}

extern "C" int glide_col2im3_f32(const float* dcol, float* dx, int Bn, int H, int W, int C, int Kp, void* stream) {
    if (!dcol || !dx) return GLIDE_E_NULL;
    if (Bn < 1 || H < 1 || W < 1 || C < 1 || Kp < 9 * C) return GLIDE_E_SHAPE;
    glide::count_launch(), glide::col2im3_k<<<glide::blocks_for(int64_t(Bn) * H * W * C), 256, 0, (cudaStream_t)stream>>>(dcol, dx, Bn, H, W,
                                                                                                   C, Kp);
    return (int)cudaGetLastError();
}

extern "C" int glide_transpose_bf16(const void* src, void* dst, int R, int Cc, void* stream) {
    if (!src || !dst) return GLIDE_E_NULL;
    if (R < 1 || Cc < 1) return GLIDE_E_SHAPE;
    dim3 grid((Cc + 31) / 32, (R + 31) / 32);
    glide::count_launch(), glide::transpose_bf16_k<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)src,
                                                                           (__nv_bfloat16*)dst, R, Cc);
    return (int)cudaGetLastError();
}
