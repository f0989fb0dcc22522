// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05 + TMEM)
// for the learned initial guess: 3x3 convolutions as GEMMs, either on an
// explicit im2col matrix (training, whose weight gradient needs it) or with
// the im2col done while staging the A tile (inference, no im2col buffer).
//
//   C[M,N] (+)= A[M,K] * B[N,K]^T   (A, B: BF16, K-major; accumulate FP32 in TMEM)
//   epilogue: + bias[N], ReLU, store FP32 or BF16, or add into FP32 C.
//
// Operands are staged in shared memory in the UMMA canonical K-major
// no-swizzle layout (8-row x 16-byte core matrices, LBO = 128 B between the
// K halves, SBO = 1024 B between 8-row groups); one elected thread issues
// four tcgen05.mma (M=128, K=16) per 64-wide K chunk into a TMEM accumulator
// and commits them to an mbarrier; the epilogue reads TMEM with tcgen05.ld
// (each warp its 32-lane subpartition).  Two kernels:
//  * tc_gemm_pipe_kernel (aligned operands, every convolution): a 2-stage
//    (short K) or 4-stage ring filled by cp.async, N tile 32/64/128 after
//    the output width;
//  * tc_gemm_kernel (any pitch or K): one 128 x 64 tile staged through
//    registers per chunk, every thread waiting for its MMAs before the next.
//
// Every wait is bounded: after ~1 s the kernel sets *err = 1, stops issuing,
// waits (bounded) for its own MMAs, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <stdint.h>

#include "glide_b200.h"

namespace glide {
void count_launch();
}

namespace glide {

constexpr int GM = 128, GN = 64, GK = 64, GTHREADS = 128;
constexpr uint32_t TMEM_COLS = 64;
constexpr long long WAIT_CYCLES = 2000000000LL;  // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory matrix descriptor, K-major, no swizzle (SM100 version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= uint64_t((saddr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;
    return d;
}

// Instruction descriptor: D = F32, A = B = BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try(addr, parity)) {
        if (clock64() - t0 > WAIT_CYCLES) return false;
    }
    return true;
}

// offset of element (row, k) inside a [rows x GK] canonical tile
__device__ __forceinline__ uint32_t tile_off(int row, int kc) {
    return uint32_t((row >> 3) * 1024 + kc * 128 + (row & 7) * 16);
}

// Stage rows [r0, r0+R) x cols [k0, k0+GK) of a K-major BF16 matrix (ld elements).
template <int R>
__device__ __forceinline__ void stage_tile(uint8_t* s, const __nv_bfloat16* __restrict__ g, int rows, int K, int ld,
                                           int r0, int k0) {
    for (int idx = threadIdx.x; idx < R * (GK / 8); idx += GTHREADS) {
        const int row = idx / (GK / 8), kc = idx % (GK / 8);
        const int gr = r0 + row, gk = k0 + kc * 8;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (gr < rows && gk < K) {
            const __nv_bfloat16* src = g + int64_t(gr) * ld + gk;
            if (gk + 8 <= K && ((reinterpret_cast<uintptr_t>(src) & 15) == 0)) {
                val = *reinterpret_cast<const uint4*>(src);
            } else {
                __nv_bfloat16 tmp[8];
#pragma unroll
                for (int e = 0; e < 8; e++) tmp[e] = (gk + e < K) ? src[e] : __float2bfloat16(0.0f);
                val = *reinterpret_cast<uint4*>(tmp);
            }
        }
        *reinterpret_cast<uint4*>(s + tile_off(row, kc)) = val;
    }
}

// Implicit im2col of a 3x3 "same" convolution: rows [m0, m0+GM) of the A
// operand are output pixels p = (b*H + y)*W + x of an NHWC BF16 input
// (C a multiple of 8, so each 16-byte chunk of a row lies in one tap), column
// k = (ky*3 + kx)*C + c holds x[b, y+ky-1, x+kx-1, c] (zero outside).  The
// staged tile is the one stage_tile would read from the explicit im2col
// matrix, so the products are bit-identical.
struct ConvShape {
    int Bn, H, W, C;
};
__device__ __forceinline__ void stage_tile_conv(uint8_t* s, const __nv_bfloat16* __restrict__ x, const ConvShape cs,
                                                int M, int K, int m0, int k0) {
    for (int idx = threadIdx.x; idx < GM * (GK / 8); idx += GTHREADS) {
        const int row = idx / (GK / 8), kc = idx % (GK / 8);
        const int p = m0 + row, k = k0 + kc * 8;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (p < M && k < K) {
            const int tap = k / cs.C, c = k - tap * cs.C;
            const int ky = tap / 3, kx = tap - 3 * ky;
            const int xx = p % cs.W, t = p / cs.W;
            const int yy = t % cs.H, b = t / cs.H;
            const int sy = yy + ky - 1, sx = xx + kx - 1;
            if (sy >= 0 && sy < cs.H && sx >= 0 && sx < cs.W)
                val = *reinterpret_cast<const uint4*>(x + ((int64_t(b) * cs.H + sy) * cs.W + sx) * cs.C + c);
        }
        *reinterpret_cast<uint4*>(s + tile_off(row, kc)) = val;
    }
}

// out_mode: 0 = store FP32, 1 = store BF16, 2 = add into FP32.  CONV: A is the
// NHWC input of a 3x3 convolution read through stage_tile_conv (lda unused).
template <bool CONV>
__global__ void __launch_bounds__(GTHREADS) tc_gemm_kernel(const __nv_bfloat16* __restrict__ A, int lda,
                                                           const __nv_bfloat16* __restrict__ B, int ldb, void* C,
                                                           int ldc, int M, int N, int K,
                                                           const float* __restrict__ bias, int relu, int out_mode,
                                                           int* err, ConvShape cs) {
    __shared__ __align__(1024) uint8_t sA[GM * GK * 2];
    __shared__ __align__(1024) uint8_t sB[GN * GK * 2];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * GN;
    const uint32_t mbar_addr = smem_u32(&mbar);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_addr));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    const uint32_t idesc = idesc_bf16_f32(GM, GN);
    const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
    uint32_t phase = 0;
    bool ok = true;
    const int nchunks = (K + GK - 1) / GK;
    for (int ch = 0; ch < nchunks && ok; ch++) {
        const int k0 = ch * GK;
        if (CONV)
            stage_tile_conv(sA, A, cs, M, K, m0, k0);
        else
            stage_tile<GM>(sA, A, M, K, lda, m0, k0);
        stage_tile<GN>(sB, B, N, K, ldb, n0, k0);
        // make the generic-proxy smem writes visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < GK / 16; s++) {
                const uint64_t da = umma_desc(a_base + s * 256, 128, 1024);
                const uint64_t db = umma_desc(b_base + s * 256, 128, 1024);
                const uint32_t acc = (ch > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             mbar_addr)
                         : "memory");
        }
        // every thread waits for the MMAs that read the staged tile; the
        // outcome is made uniform so all threads leave the loop together
        const int mine = mbar_wait_bounded(mbar_addr, phase) ? 1 : 0;
        ok = __syncthreads_and(mine) != 0;
        if (!ok) break;
        phase ^= 1u;
    }
    if (!ok) {
        if (threadIdx.x == 0 && err) atomicExch(err, 1);
        mbar_wait_bounded(mbar_addr, phase);   // bounded drain of the MMAs still in flight
        __syncthreads();
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (ok && nchunks > 0) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < GN; c0 += 8) {
            uint32_t r[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "r"(taddr + uint32_t(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int col = n0 + c0 + e;
                    if (col >= N) continue;
                    float x = __uint_as_float(r[e]);
                    if (bias) x += bias[col];
                    if (relu) x = fmaxf(x, 0.0f);
                    const int64_t o = int64_t(row) * ldc + col;
                    if (out_mode == 0) reinterpret_cast<float*>(C)[o] = x;
                    else if (out_mode == 1) reinterpret_cast<__nv_bfloat16*>(C)[o] = __float2bfloat16(x);
                    else reinterpret_cast<float*>(C)[o] += x;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// --------------------------------------------------------------------------
// Pipelined form (what aligned GEMMs and every convolution run): a ring of
// PSTAGES shared-memory stages filled by 16-byte cp.async copies (zero-filled
// outside the matrix or the image, so the implicit im2col needs no branch
// around the copy), so the copies of the next chunks are in flight while the
// tensor core works on the current one.  Chunk c lives in stage c % PSTAGES;
// before a stage is refilled its previous chunk's MMAs must have completed
// (their tcgen05.commit arrives on that stage's mbarrier).  The thread ->
// chunk map is fixed (kc = thread % 8, rows thread / 8 + 16 i), so the
// per-row pixel decomposition of the convolution is done once per CTA and a
// K chunk costs one division per thread.  The N tile (32, 64 or 128) follows
// the output width, so narrow layers issue narrow MMAs and wide ones stage A
// once for 128 outputs.  The epilogue stores 8 BF16 outputs per 16-byte
// store where the row allows it.
// --------------------------------------------------------------------------
constexpr int PSTAGES_MAX = 4;

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <bool CONV, int BN, int PSTAGES>
__global__ void __launch_bounds__(GTHREADS) tc_gemm_pipe_kernel(const __nv_bfloat16* __restrict__ A, int lda,
                                                                const __nv_bfloat16* __restrict__ B, int ldb,
                                                                void* C, int ldc, int M, int N, int K,
                                                                const float* __restrict__ bias, int relu,
                                                                int out_mode, int* err, ConvShape cs) {
    constexpr int A_BYTES = GM * GK * 2, B_BYTES = BN * GK * 2, STAGE = A_BYTES + B_BYTES;
    constexpr int AROWS = GM / 16, BROWS = BN / 16;   // rows per thread and chunk
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar[PSTAGES_MAX];
    __shared__ uint32_t tmem_slot;

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * BN;
    const int kc = threadIdx.x & 7, rsub = threadIdx.x >> 3;
    const uint32_t sbase = (smem_u32(smem) + 1023u) & ~1023u;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(uint32_t(BN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < PSTAGES; s++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[s])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    // per-row state of this thread's A rows
    int64_t a_off[AROWS];      // CONV: pixel index; GEMM: row offset in elements
    int a_y[AROWS], a_x[AROWS];
    bool a_ok[AROWS];
#pragma unroll
    for (int i = 0; i < AROWS; i++) {
        const int p = m0 + rsub + 16 * i;
        a_ok[i] = p < M;
        if (CONV) {
            const int pp = a_ok[i] ? p : 0;
            const int xx = pp % cs.W, t = pp / cs.W;
            a_x[i] = xx;
            a_y[i] = t % cs.H;
            a_off[i] = int64_t(pp);
        } else {
            a_x[i] = a_y[i] = 0;
            a_off[i] = int64_t(a_ok[i] ? p : 0) * lda;
        }
    }

    const int nchunks = (K + GK - 1) / GK;
    auto issue_chunk = [&](int ch) {
        const uint32_t st = sbase + uint32_t((ch % PSTAGES) * STAGE);
        const int k = ch * GK + kc * 8;
        const bool kin = k < K;
        if (CONV) {
            int dy = 0, dx = 0, c = 0;
            if (kin) {
                const int tap = k / cs.C;
                c = k - tap * cs.C;
                const int ky = tap / 3;
                dy = ky - 1;
                dx = tap - 3 * ky - 1;
            }
            const int64_t doff = (int64_t(dy) * cs.W + dx) * cs.C + c;
#pragma unroll
            for (int i = 0; i < AROWS; i++) {
                const int sy = a_y[i] + dy, sx = a_x[i] + dx;
                const bool ok = kin && a_ok[i] && sy >= 0 && sy < cs.H && sx >= 0 && sx < cs.W;
                const __nv_bfloat16* src = ok ? A + a_off[i] * cs.C + doff : A;
                cp_async16(st + tile_off(rsub + 16 * i, kc), src, ok ? 16u : 0u);
            }
        } else {
#pragma unroll
            for (int i = 0; i < AROWS; i++) {
                const bool ok = kin && a_ok[i];
                cp_async16(st + tile_off(rsub + 16 * i, kc), ok ? A + a_off[i] + k : A, ok ? 16u : 0u);
            }
        }
#pragma unroll
        for (int i = 0; i < BROWS; i++) {
            const int n = n0 + rsub + 16 * i;
            const bool ok = kin && n < N;
            cp_async16(st + A_BYTES + tile_off(rsub + 16 * i, kc), ok ? B + int64_t(n) * ldb + k : B, ok ? 16u : 0u);
        }
    };

#pragma unroll
    for (int s = 0; s < PSTAGES - 1; s++) {
        if (s < nchunks) issue_chunk(s);
        cp_async_commit();
    }
    const uint32_t idesc = idesc_bf16_f32(GM, BN);
    bool ok = true;
    int issued = 0;   // chunks whose MMAs were issued
    for (int ch = 0; ch < nchunks; ch++) {
        // refill the stage of chunk ch-1 with chunk ch+PSTAGES-1 once chunk ch-1's MMAs are done
        const int nxt = ch + PSTAGES - 1;
        if (ch >= 1 && nxt < nchunks) {
            const int pc = ch - 1;
            const int mine = mbar_wait_bounded(smem_u32(&mbar[pc % PSTAGES]), uint32_t((pc / PSTAGES) & 1)) ? 1 : 0;
            ok = __syncthreads_and(mine) != 0;
            if (!ok) break;
        }
        if (nxt < nchunks) issue_chunk(nxt);
        cp_async_commit();
        cp_async_wait<PSTAGES - 1>();     // this thread's copies of chunk ch have landed
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();                  // ... and every thread's
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = sbase + uint32_t((ch % PSTAGES) * STAGE);
#pragma unroll
            for (int s = 0; s < GK / 16; s++) {
                const uint64_t da = umma_desc(st + s * 256, 128, 1024);
                const uint64_t db = umma_desc(st + A_BYTES + s * 256, 128, 1024);
                const uint32_t acc = (ch > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    :
                    : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar[ch % PSTAGES]))
                         : "memory");
        }
        issued = ch + 1;
    }
    cp_async_wait<0>();
    // MMAs complete in issue order: the last commit covers every chunk
    if (issued > 0) {
        const int pc = issued - 1;
        const int mine = mbar_wait_bounded(smem_u32(&mbar[pc % PSTAGES]), uint32_t((pc / PSTAGES) & 1)) ? 1 : 0;
        const bool done = __syncthreads_and(mine) != 0;
        ok = ok && done;
    }
    if (!ok && threadIdx.x == 0 && err) atomicExch(err, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (ok && issued == nchunks && nchunks > 0) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16);
        const bool vec = out_mode == 1 && (ldc & 7) == 0 && (reinterpret_cast<uintptr_t>(C) & 15) == 0;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 8) {
            uint32_t r[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "r"(taddr + uint32_t(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int col0 = n0 + c0;
            if (row >= M || col0 >= N) continue;
            float x[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                x[e] = __uint_as_float(r[e]);
                if (bias && col0 + e < N) x[e] += bias[col0 + e];
                if (relu) x[e] = fmaxf(x[e], 0.0f);
            }
            const int64_t o = int64_t(row) * ldc + col0;
            if (vec && col0 + 8 <= N) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int e = 0; e < 8; e++) h[e] = __float2bfloat16(x[e]);
                *reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(C) + o) = *reinterpret_cast<uint4*>(h);
                continue;
            }
#pragma unroll
            for (int e = 0; e < 8; e++) {
                if (col0 + e >= N) break;
                if (out_mode == 0) reinterpret_cast<float*>(C)[o + e] = x[e];
                else if (out_mode == 1) reinterpret_cast<__nv_bfloat16*>(C)[o + e] = __float2bfloat16(x[e]);
                else reinterpret_cast<float*>(C)[o + e] += x[e];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(BN)));
    }
}

template <bool CONV, int BN, int PSTAGES>
int launch_pipe(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, void* C, int ldc, int M, int N,
                int K, const float* bias, int relu, int out_mode, int* err, ConvShape cs, cudaStream_t s) {
    constexpr int SMEM = PSTAGES * (GM * GK * 2 + BN * GK * 2) + 1024;
    static int configured[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return GLIDE_E_SHAPE;
    if (!configured[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(tc_gemm_pipe_kernel<CONV, BN, PSTAGES>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
        if (e != cudaSuccess) return int(e);
        configured[dev] = 1;
    }
    dim3 grid((M + GM - 1) / GM, (N + BN - 1) / BN);
    count_launch(), tc_gemm_pipe_kernel<CONV, BN, PSTAGES><<<grid, GTHREADS, SMEM, s>>>(
        A, lda, B, ldb, C, ldc, M, N, K, bias, relu, out_mode, err, cs);
    return int(cudaGetLastError());
}

// Short K (a few chunks, the convolutions of the guess network) runs a
// 2-stage ring: half the shared memory, so 2-3x the CTAs per SM hide each
// CTA's fixed latencies (ncu at 1024^2, C = 32, 4 stages: 2 CTAs and 7.7
// warps per SM, tensor pipe 3 % active); long K keeps 4 stages.
template <bool CONV, int BN>
int launch_pipe_s(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, void* C, int ldc, int M, int N,
                  int K, const float* bias, int relu, int out_mode, int* err, ConvShape cs, cudaStream_t s) {
    if ((K + GK - 1) / GK <= 8)
        return launch_pipe<CONV, BN, 2>(A, lda, B, ldb, C, ldc, M, N, K, bias, relu, out_mode, err, cs, s);
    return launch_pipe<CONV, BN, 4>(A, lda, B, ldb, C, ldc, M, N, K, bias, relu, out_mode, err, cs, s);
}

template <bool CONV>
int launch_pipe_n(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, void* C, int ldc, int M, int N,
                  int K, const float* bias, int relu, int out_mode, int* err, ConvShape cs, cudaStream_t s) {
    if (N <= 32) return launch_pipe_s<CONV, 32>(A, lda, B, ldb, C, ldc, M, N, K, bias, relu, out_mode, err, cs, s);
    if (N <= 64) return launch_pipe_s<CONV, 64>(A, lda, B, ldb, C, ldc, M, N, K, bias, relu, out_mode, err, cs, s);
    return launch_pipe_s<CONV, 128>(A, lda, B, ldb, C, ldc, M, N, K, bias, relu, out_mode, err, cs, s);
}

inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace glide

extern "C" int glide_gemm_bf16(const void* A, int lda, const void* B, int ldb, void* C, int ldc, int M, int N, int K,
                               const float* bias, int relu, int out_mode, int* err, void* stream) {
    if (!A || !B || !C) return GLIDE_E_NULL;
    if (M < 1 || N < 1 || K < 1 || lda < K || ldb < K || ldc < N || out_mode < 0 || out_mode > 2) return GLIDE_E_SHAPE;
    if (K % 8 == 0 && lda % 8 == 0 && ldb % 8 == 0 && glide::al16(A) && glide::al16(B))
        return glide::launch_pipe_n<false>((const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, C, ldc, M, N, K,
                                           bias, relu, out_mode, err, glide::ConvShape{0, 0, 0, 0},
                                           (cudaStream_t)stream);
    dim3 grid((M + glide::GM - 1) / glide::GM, (N + glide::GN - 1) / glide::GN);
    glide::count_launch(), glide::tc_gemm_kernel<false><<<grid, glide::GTHREADS, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, C, ldc, M, N, K, bias, relu, out_mode, err,
        glide::ConvShape{0, 0, 0, 0});
    return (int)cudaGetLastError();
}

extern "C" int glide_conv3x3_bf16(const void* x, int Bn, int H, int W, int C, const void* Wt, int ldw, void* out,
                                  int ldc, int N, const float* bias, int relu, int out_mode, int* err, void* stream) {
    if (!x || !Wt || !out) return GLIDE_E_NULL;
    if (Bn < 1 || H < 1 || W < 1 || C < 8 || C % 8 != 0 || N < 1 || ldw < 9 * C || ldc < N || out_mode < 0 ||
        out_mode > 2)
        return GLIDE_E_SHAPE;
    if ((reinterpret_cast<uintptr_t>(x) & 15) != 0) return GLIDE_E_SHAPE;
    const int64_t M64 = int64_t(Bn) * H * W;
    if (M64 >= (int64_t(1) << 31)) return GLIDE_E_TOO_LARGE;
    const int M = int(M64), K = 9 * C;
    if (ldw % 8 == 0 && glide::al16(Wt))
        return glide::launch_pipe_n<true>((const __nv_bfloat16*)x, 0, (const __nv_bfloat16*)Wt, ldw, out, ldc, M, N, K,
                                          bias, relu, out_mode, err, glide::ConvShape{Bn, H, W, C},
                                          (cudaStream_t)stream);
    dim3 grid((M + glide::GM - 1) / glide::GM, (N + glide::GN - 1) / glide::GN);
    glide::count_launch(), glide::tc_gemm_kernel<true><<<grid, glide::GTHREADS, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)x, 0, (const __nv_bfloat16*)Wt, ldw, out, ldc, M, N, K, bias, relu, out_mode, err,
        glide::ConvShape{Bn, H, W, C});
    return (int)cudaGetLastError();
}
