// Vanka sweeps without caller-provided scratch: glide_vanka_sweeps_noalloc.
//
// glide_vanka_sweeps needs a scratch buffer of 5 * ny * nx * nb elements for
// the per-cell Newton deltas, which the caller allocates.  Some callers cannot
// call cudaMalloc: a host whose memory pool owns all device memory and hands a
// plugin only its input and output buffers, or a latency-critical loop that
// must not hit cudaMalloc's implicit device synchronisation.  For them this
// entry point keeps the scratch in a file-scope device array of fixed size,
// which every GPU that loads the library holds until the process exits.
//
// Limits and behaviour:
//  * capacity: NOALLOC_SCRATCH_BYTES = 10 MiB, i.e. 5 deltas per cell for at
//    most 262,144 cells (nb * ny * nx) in FP64 or 524,288 cells in FP32;
//    larger problems are rejected with GLIDE_E_TOO_LARGE before any launch;
//  * the device address of the array is looked up once per device, on the
//    first call made with that device current (cudaGetSymbolAddress); make
//    that first call before any stream capture on that device;
//  * all calls share the one array: calls that overlap on the GPU (other
//    streams, other host threads) race on it and must be ordered by the
//    caller; the array keeps the last call's contents, and nothing needs
//    clearing because every value a sweep reads is written earlier in the
//    same sweep;
//  * no cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>

#include <mutex>

#include "glide_b200.h"

namespace glide {
template <typename T>
int launch_vanka_sweeps(const GlideLevelArgs*, const void*, const void*, const void*, int, int, double, double,
                        const int*, const int*, void*, cudaStream_t, double, int);
}

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(10) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
void* g_scratch_ptr[MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device (set-up on the
// first call per device).  In host code the symbol itself is only a host-side
// stand-in, so the address must come from cudaGetSymbolAddress.
int scratch_address(void** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return int(e);
    if (dev < 0 || dev >= MAX_DEVICES) return GLIDE_E_SHAPE;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return int(e);
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return 0;
}

}  // namespace

extern "C" size_t glide_noalloc_scratch_bytes(void) { return NOALLOC_SCRATCH_BYTES; }

extern "C" int glide_vanka_sweeps_noalloc(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H,
                                          int n_iter, int n_newton, double omega, double shift, const int* flags,
                                          const int* any_active, void* stream) {
    if (!a || !f_u || !f_v || !f_H) return GLIDE_E_NULL;
    if (a->dtype != GLIDE_F32 && a->dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (a->ny < 1 || a->nx < 1 || a->nb < 1 || n_iter < 0 || n_newton < 0) return GLIDE_E_SHAPE;
    if (!a->u || !a->v || !a->H || !a->bed || !a->B || !a->beta || !a->mask || !a->gamma) return GLIDE_E_NULL;
    if ((flags == nullptr) != (any_active == nullptr)) return GLIDE_E_NULL;
    const size_t elem = a->dtype == GLIDE_F32 ? 4 : 8;
    const size_t need = size_t(5) * size_t(a->nb) * size_t(a->ny) * size_t(a->nx) * elem;
    if (need > NOALLOC_SCRATCH_BYTES) return GLIDE_E_TOO_LARGE;
    void* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    return a->dtype == GLIDE_F32
               ? glide::launch_vanka_sweeps<float>(a, f_u, f_v, f_H, n_iter, n_newton, omega, shift, flags, any_active,
                                                   scratch, (cudaStream_t)stream, GLIDE_REF_NEWTON_STEP, 0)
               : glide::launch_vanka_sweeps<double>(a, f_u, f_v, f_H, n_iter, n_newton, omega, shift, flags,
                                                    any_active, scratch, (cudaStream_t)stream, GLIDE_REF_NEWTON_STEP, 0);
}
