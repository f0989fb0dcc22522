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
//  * the device address of the array is looked up on the first call made
//    with a device current (cudaGetSymbolAddress) and cached together with
//    the unique id of the CUDA context it belongs to; a later call in another
//    context of that device (after cudaDeviceReset, or once the primary
//    context was released and created again, when the library's module and
//    so the array may have moved) looks it up again.  Make the first call on
//    a device, and the first call after such a reset, before any stream
//    capture on that device;
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
struct Cached {
    unsigned long long ctx_id;  // unique id of the context the address belongs to (cuCtxGetId)
    void* ptr;
};
Cached g_cache[MAX_DEVICES] = {};

// Driver queries reached through the runtime (no link against libcuda):
// CUresult cuCtxGetCurrent(CUcontext*), CUresult cuCtxGetId(CUcontext, unsigned long long*).
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
std::once_flag g_entry_once;

void load_entry_points() {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
}

// Id of the context current on this thread; 0 if there is none (or it
// cannot be queried, in which case the address is looked up every call).
unsigned long long current_ctx_id() {
    std::call_once(g_entry_once, load_entry_points);
    if (!g_ctx_current || !g_ctx_id) return 0;
    void* ctx = nullptr;
    if (g_ctx_current(&ctx) != 0 || ctx == nullptr) return 0;
    unsigned long long id = 0;
    if (g_ctx_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array in the current context.  In host code
// the symbol itself is only a host-side stand-in, so the address must come
// from cudaGetSymbolAddress.
int scratch_address(void** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return int(e);
    if (dev < 0 || dev >= MAX_DEVICES) return GLIDE_E_SHAPE;
    std::lock_guard<std::mutex> lock(g_mutex);
    Cached& c = g_cache[dev];
    const unsigned long long id = current_ctx_id();
    if (c.ptr != nullptr && id != 0 && id == c.ctx_id) {
        *out = c.ptr;
        return 0;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // also creates the context on a first call
    if (e != cudaSuccess) return int(e);
    c.ptr = p;
    c.ctx_id = id != 0 ? id : current_ctx_id();
    *out = p;
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
