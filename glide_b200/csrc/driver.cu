// C ABI dispatch and the native multigrid drivers.
//
// glide_fascd_vcycle / glide_adjoint_vcycle restate the call sequences of
// glide/solver.py:71-220 as device-side launches on one stream (no host
// synchronisation inside a cycle), so a whole cycle can be captured once into
// a CUDA graph and replayed (glide_graph_*).
#include <atomic>
#include <cstdio>
#include <cstring>
#include <vector>

#include "glide_common.cuh"

namespace glide {
static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_total() { return g_launches.load(std::memory_order_relaxed); }

template <typename T> int launch_residual(const GlideLevelArgs*, const void*, const void*, const void*, void*, void*, void*, cudaStream_t);
template <typename T>
int launch_jvp(const GlideLevelArgs*, const void*, const void*, const void*, const void*, const void*, const void*,
               void*, void*, void*, cudaStream_t);
template <typename T> int launch_vjp(const GlideLevelArgs*, const void*, const void*, const void*, const void*, const void*, const void*, void*, void*, void*, int, cudaStream_t);
template <typename T> int launch_grad_beta(const GlideLevelArgs*, const void*, const void*, void*, int, cudaStream_t);
template <typename T> int launch_vanka_sweeps(const GlideLevelArgs*, const void*, const void*, const void*, int, int, double, double, const int*, const int*, void*, cudaStream_t, double, int);
template <typename T> int launch_vanka_lu(const GlideLevelArgs*, const void*, void*, double, cudaStream_t);
template <typename T> int launch_vanka_linear(const GlideLevelArgs*, const void*, const void*, const void*, const void*, void*, void*, void*, double, void*, cudaStream_t);
template <typename T> int launch_vanka_cells(const GlideLevelArgs*, const void*, const void*, const void*, int, int, double, const int*, const int*, void*, cudaStream_t, double);
template <typename T> int launch_error_mask(const GlideLevelArgs*, const void*, const void*, const void*, double, void*, int*, int*, cudaStream_t);
template <typename T> int launch_tile_flags(const GlideLevelArgs*, const void*, int*, int*, cudaStream_t);
template <typename T> int launch_vanka_adjoint(const GlideLevelArgs*, void*, void*, void*, const void*, const void*, const void*, int, double, cudaStream_t);
template <typename T> int launch_restrict(int, int, const void*, void*, int, int, int, cudaStream_t);
template <typename T> int launch_prolong(int, int, int, const void*, void*, int, int, int, cudaStream_t);
template <typename T> int launch_lincomb(void*, const void*, double, const void*, double, int64_t, cudaStream_t);
template <typename T> int launch_fill(void*, double, int64_t, cudaStream_t);
template <typename T> int launch_mask_le(void*, const void*, const void*, double, int64_t, cudaStream_t);
template <typename T> int launch_constraint_down(void*, void*, const void*, const void*, int, int, int, cudaStream_t);
template <typename T> int launch_norms(double*, double*, const void*, const void*, const void*, const void*, const void*, int64_t, int64_t, int64_t, cudaStream_t);
template <typename T> int launch_axpy_dev(void*, const void*, const double*, const void*, int64_t, cudaStream_t);
int launch_ls_pick(double*, const double*, int, cudaStream_t);
int norms_parts_count(int64_t n);

template <typename D, typename S>
__global__ void convert_k(D* __restrict__ out, const S* __restrict__ x, int64_t n, int acc) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n) return;
    D v = D(x[k]);
    out[k] = acc ? out[k] + v : v;
}
}  // namespace glide

using namespace glide;

static inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

static int check_level(const GlideLevelArgs* a) {
    if (!a) return GLIDE_E_NULL;
    if (a->dtype != GLIDE_F32 && a->dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (a->ny < 1 || a->nx < 1 || a->nb < 1) return GLIDE_E_SHAPE;
    // the stencil and smoother kernels index one problem's fields with 32-bit
    // element offsets (the largest field, (ny+1)(nx+1), far exceeds HBM first)
    if (int64_t(a->ny + 1) * (a->nx + 1) >= (int64_t(1) << 31)) return GLIDE_E_TOO_LARGE;
    if (!a->u || !a->v || !a->H || !a->bed || !a->B || !a->beta || !a->mask || !a->gamma) return GLIDE_E_NULL;
    return GLIDE_OK;
}

#define TDISPATCH(dtype, call_f32, call_f64) \
    ((dtype) == GLIDE_F32 ? (call_f32) : (call_f64))

extern "C" {

const char* glide_version(void) { return "glide_b200 0.1 (sm_100a)"; }

long long glide_launch_count(void) { return glide::launch_total(); }

int glide_residual(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, void* r_u, void* r_v,
                   void* r_H, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!f_u || !f_v || !f_H || !r_u || !r_v || !r_H) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype, launch_residual<float>(a, f_u, f_v, f_H, r_u, r_v, r_H, S(stream)),
                     launch_residual<double>(a, f_u, f_v, f_H, r_u, r_v, r_H, S(stream)));
}

int glide_jvp(const GlideLevelArgs* a, const void* d_u, const void* d_v, const void* d_H, void* j_u, void* j_v,
              void* j_H, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!d_u || !d_v || !d_H || !j_u || !j_v || !j_H) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype,
                     launch_jvp<float>(a, d_u, d_v, d_H, nullptr, nullptr, nullptr, j_u, j_v, j_H, S(stream)),
                     launch_jvp<double>(a, d_u, d_v, d_H, nullptr, nullptr, nullptr, j_u, j_v, j_H, S(stream)));
}

int glide_jvp_add(const GlideLevelArgs* a, const void* d_u, const void* d_v, const void* d_H, const void* base_u,
                  const void* base_v, const void* base_H, void* out_u, void* out_v, void* out_H, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!d_u || !d_v || !d_H || !base_u || !base_v || !base_H || !out_u || !out_v || !out_H) return GLIDE_E_NULL;
    if (out_u == base_u || out_v == base_v || out_H == base_H || out_u == d_u || out_v == d_v || out_H == d_H)
        return GLIDE_E_SHAPE;
    return TDISPATCH(a->dtype,
                     launch_jvp<float>(a, d_u, d_v, d_H, base_u, base_v, base_H, out_u, out_v, out_H, S(stream)),
                     launch_jvp<double>(a, d_u, d_v, d_H, base_u, base_v, base_H, out_u, out_v, out_H, S(stream)));
}

int glide_vjp(const GlideLevelArgs* a, const void* l_u, const void* l_v, const void* l_H, const void* f_u,
              const void* f_v, const void* f_H, void* o_u, void* o_v, void* o_H, int exact_boundary, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!l_u || !l_v || !l_H || !o_u || !o_v || !o_H) return GLIDE_E_NULL;
    if ((f_u != nullptr) != (f_v != nullptr) || (f_u != nullptr) != (f_H != nullptr)) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype,
                     launch_vjp<float>(a, l_u, l_v, l_H, f_u, f_v, f_H, o_u, o_v, o_H, exact_boundary, S(stream)),
                     launch_vjp<double>(a, l_u, l_v, l_H, f_u, f_v, f_H, o_u, o_v, o_H, exact_boundary, S(stream)));
}

int glide_grad_beta(const GlideLevelArgs* a, const void* l_u, const void* l_v, void* grad, int exact_boundary,
                    void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!l_u || !l_v || !grad) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype, launch_grad_beta<float>(a, l_u, l_v, grad, exact_boundary, S(stream)),
                     launch_grad_beta<double>(a, l_u, l_v, grad, exact_boundary, S(stream)));
}

int glide_vanka_sweeps_ex(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_iter,
                          int n_newton, double newton_step, double omega, double shift, int pivoted_lu,
                          const int* flags, const int* any_active, void* scratch, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!f_u || !f_v || !f_H || !scratch) return GLIDE_E_NULL;
    if ((flags == nullptr) != (any_active == nullptr)) return GLIDE_E_NULL;
    if (n_iter < 0 || n_newton < 0 || !(newton_step > 0.0 && newton_step <= 1.0)) return GLIDE_E_SHAPE;
    const int pv = pivoted_lu ? 1 : 0;
    return TDISPATCH(a->dtype,
                     launch_vanka_sweeps<float>(a, f_u, f_v, f_H, n_iter, n_newton, omega, shift, flags, any_active,
                                                scratch, S(stream), newton_step, pv),
                     launch_vanka_sweeps<double>(a, f_u, f_v, f_H, n_iter, n_newton, omega, shift, flags,
                                                 any_active, scratch, S(stream), newton_step, pv));
}

int glide_vanka_sweeps(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_iter,
                       int n_newton, double omega, double shift, const int* flags, const int* any_active,
                       void* scratch, void* stream) {
    return glide_vanka_sweeps_ex(a, f_u, f_v, f_H, n_iter, n_newton, GLIDE_REF_NEWTON_STEP, omega, shift, 0, flags,
                                 any_active, scratch, stream);
}

int glide_vanka_lu(const GlideLevelArgs* a, const void* f_H, void* lu, double shift, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!lu || !f_H) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype, launch_vanka_lu<float>(a, f_H, lu, shift, S(stream)),
                     launch_vanka_lu<double>(a, f_H, lu, shift, S(stream)));
}

int glide_vanka_lu_masked(const GlideLevelArgs* a, void* lu, double shift, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!lu) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype, launch_vanka_lu<float>(a, nullptr, lu, shift, S(stream)),
                     launch_vanka_lu<double>(a, nullptr, lu, shift, S(stream)));
}

int glide_vanka_linear(const GlideLevelArgs* a, const void* rho_u, const void* rho_v, const void* rho_H,
                       const void* lu, void* d_u, void* d_v, void* d_H, double omega, void* scratch, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!rho_u || !rho_v || !rho_H || !lu || !d_u || !d_v || !d_H || !scratch) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype,
                     launch_vanka_linear<float>(a, rho_u, rho_v, rho_H, lu, d_u, d_v, d_H, omega, scratch, S(stream)),
                     launch_vanka_linear<double>(a, rho_u, rho_v, rho_H, lu, d_u, d_v, d_H, omega, scratch,
                                                 S(stream)));
}

int glide_vanka_cells(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_launch,
                      int n_newton, double shift, const int* flags, const int* any_active, void* scratch,
                      void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!f_u || !f_v || !f_H || !scratch) return GLIDE_E_NULL;
    if ((flags == nullptr) != (any_active == nullptr)) return GLIDE_E_NULL;
    if (n_launch < 0 || n_newton < 0) return GLIDE_E_SHAPE;
    return TDISPATCH(a->dtype,
                     launch_vanka_cells<float>(a, f_u, f_v, f_H, n_launch, n_newton, shift, flags, any_active,
                                               scratch, S(stream), GLIDE_REF_NEWTON_STEP),
                     launch_vanka_cells<double>(a, f_u, f_v, f_H, n_launch, n_newton, shift, flags, any_active,
                                                scratch, S(stream), GLIDE_REF_NEWTON_STEP));
}

int glide_error_mask(const GlideLevelArgs* a, const void* r_u, const void* r_v, const void* r_H, double threshold,
                     void* err_mask, int* flags, int* any_active, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!r_u || !r_v || !r_H || !err_mask) return GLIDE_E_NULL;
    if ((flags == nullptr) != (any_active == nullptr)) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype,
                     launch_error_mask<float>(a, r_u, r_v, r_H, threshold, err_mask, flags, any_active, S(stream)),
                     launch_error_mask<double>(a, r_u, r_v, r_H, threshold, err_mask, flags, any_active, S(stream)));
}

int glide_tile_flags(const GlideLevelArgs* a, const void* err_mask, int* flags, int* any_active, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!err_mask || !flags || !any_active) return GLIDE_E_NULL;
    return TDISPATCH(a->dtype, launch_tile_flags<float>(a, err_mask, flags, any_active, S(stream)),
                     launch_tile_flags<double>(a, err_mask, flags, any_active, S(stream)));
}

int glide_vanka_adjoint(const GlideLevelArgs* a, void* l_u, void* l_v, void* l_H, const void* ra_u, const void* ra_v,
                        const void* ra_H, int color, double omega, void* stream) {
    int e = check_level(a);
    if (e) return e;
    if (!l_u || !l_v || !l_H || !ra_u || !ra_v || !ra_H) return GLIDE_E_NULL;
    if (color != 0 && color != 1) return GLIDE_E_SHAPE;
    return TDISPATCH(a->dtype, launch_vanka_adjoint<float>(a, l_u, l_v, l_H, ra_u, ra_v, ra_H, color, omega, S(stream)),
                     launch_vanka_adjoint<double>(a, l_u, l_v, l_H, ra_u, ra_v, ra_H, color, omega, S(stream)));
}

int glide_restrict(int dtype, int field, int use_max, const void* fine, void* coarse, int nyc, int nxc, int nb,
                   void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!fine || !coarse) return GLIDE_E_NULL;
    if (field < 0 || field > 2 || nyc < 1 || nxc < 1 || nb < 1) return GLIDE_E_SHAPE;
    return TDISPATCH(dtype, launch_restrict<float>(field, use_max, fine, coarse, nyc, nxc, nb, S(stream)),
                     launch_restrict<double>(field, use_max, fine, coarse, nyc, nxc, nb, S(stream)));
}

int glide_prolong(int dtype, int field, int smooth, int add, const void* coarse, void* fine, int nyc, int nxc, int nb,
                  void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!fine || !coarse) return GLIDE_E_NULL;
    if (field < 0 || field > 2 || nyc < 1 || nxc < 1 || nb < 1) return GLIDE_E_SHAPE;
    return TDISPATCH(dtype, launch_prolong<float>(field, smooth, add, coarse, fine, nyc, nxc, nb, S(stream)),
                     launch_prolong<double>(field, smooth, add, coarse, fine, nyc, nxc, nb, S(stream)));
}

int glide_lincomb(int dtype, void* out, const void* x, double a, const void* y, double b, int64_t n, void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!out || !x) return GLIDE_E_NULL;
    return TDISPATCH(dtype, launch_lincomb<float>(out, x, a, y, b, n, S(stream)),
                     launch_lincomb<double>(out, x, a, y, b, n, S(stream)));
}

int glide_fill(int dtype, void* out, double val, int64_t n, void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!out) return GLIDE_E_NULL;
    return TDISPATCH(dtype, launch_fill<float>(out, val, n, S(stream)), launch_fill<double>(out, val, n, S(stream)));
}

int glide_mask_le(int dtype, void* mask, const void* H, const void* gamma, double tol, int64_t n, void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!mask || !H || !gamma) return GLIDE_E_NULL;
    return TDISPATCH(dtype, launch_mask_le<float>(mask, H, gamma, tol, n, S(stream)),
                     launch_mask_le<double>(mask, H, gamma, tol, n, S(stream)));
}

int glide_convert(int dst_dtype, void* out, const void* x, int64_t n, int accumulate, void* stream) {
    if (dst_dtype != GLIDE_F32 && dst_dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!out || !x) return GLIDE_E_NULL;
    if (n <= 0) return GLIDE_OK;
    unsigned nb = unsigned((n + 255) / 256);
    glide::count_launch();
    if (dst_dtype == GLIDE_F32) convert_k<float, double><<<nb, 256, 0, S(stream)>>>((float*)out, (const double*)x, n, accumulate);
    else convert_k<double, float><<<nb, 256, 0, S(stream)>>>((double*)out, (const float*)x, n, accumulate);
    return (int)cudaGetLastError();
}

int glide_norm_parts(int64_t n) { return norms_parts_count(n); }

int glide_norms(int dtype, double* out3, double* parts, const void* r_u, const void* r_v, const void* r_H,
                const void* H, const void* gamma, int64_t nu, int64_t nv, int64_t nc, void* stream) {
    if (dtype != GLIDE_F32 && dtype != GLIDE_F64) return GLIDE_E_DTYPE;
    if (!out3 || !parts || !r_u || !r_v || !r_H || !H || !gamma) return GLIDE_E_NULL;
    return TDISPATCH(dtype, launch_norms<float>(out3, parts, r_u, r_v, r_H, H, gamma, nu, nv, nc, S(stream)),
                     launch_norms<double>(out3, parts, r_u, r_v, r_H, H, gamma, nu, nv, nc, S(stream)));
}

}  // extern "C"

// --------------------------------------------------------------------------
// V-cycles
// --------------------------------------------------------------------------
namespace {

struct LevelView {
    GlideLevel* L;
    int dt;
    int64_t nu, nv, nc, ntot;  // per problem
    int nb;
    void* at(void* base, int64_t off) const {
        return (char*)base + off * (dt == GLIDE_F32 ? 4 : 8);
    }
    // monolithic vector parts; a batch of nb problems stores [u|v|H] per problem
    void* u(void* V) const { return V; }
    void* v(void* V) const { return at(V, nu * nb); }
    void* H(void* V) const { return at(V, (nu + nv) * nb); }
};

LevelView view(GlideLevel* L) {
    LevelView w;
    w.L = L;
    w.dt = L->a.dtype;
    w.nb = L->a.nb;
    w.nu = int64_t(L->a.ny) * (L->a.nx + 1);
    w.nv = int64_t(L->a.ny + 1) * L->a.nx;
    w.nc = int64_t(L->a.ny) * L->a.nx;
    w.ntot = w.nu + w.nv + w.nc;
    return w;
}

#define TRY(x)                  \
    do {                        \
        int _e = (x);           \
        if (_e) return _e;      \
    } while (0)

int vanka(GlideLevel* L, int n_iter, const GlideSolverConfig* c, bool local, void* s) {
    LevelView w = view(L);
    const double step = c->newton_step > 0.0 ? c->newton_step : GLIDE_REF_NEWTON_STEP;
    return glide_vanka_sweeps_ex(&L->a, w.u(L->f), w.v(L->f), w.H(L->f), n_iter, c->n_newton, step, c->omega,
                                 c->shift, c->pivoted_lu, local ? L->flags : nullptr, local ? L->any_active : nullptr,
                                 L->scratch, s);
}

int fill_gamma(GlideLevel* L, double val, void* s) {
    LevelView w = view(L);
    return glide_fill(w.dt, (void*)L->a.gamma, val, w.nc * w.nb, s);
}

// gamma = w_H + x
int gamma_from(GlideLevel* L, const void* x, void* s) {
    LevelView w = view(L);
    return glide_lincomb(w.dt, (void*)L->a.gamma, w.H(L->w), 1.0, x, 1.0, w.nc * w.nb, s);
}

int restrict3(GlideLevel* L, GlideLevel* C, void* Vf, void* Vc, void* s) {
    LevelView wf = view(L), wc = view(C);
    int nyc = C->a.ny, nxc = C->a.nx, nb = C->a.nb;
    TRY(glide_restrict(wf.dt, 0, 0, wf.u(Vf), wc.u(Vc), nyc, nxc, nb, s));
    TRY(glide_restrict(wf.dt, 1, 0, wf.v(Vf), wc.v(Vc), nyc, nxc, nb, s));
    TRY(glide_restrict(wf.dt, 2, 0, wf.H(Vf), wc.H(Vc), nyc, nxc, nb, s));
    return 0;
}

// U = U_pre + a * P(U_c - w_c), a from GLIDE_LS_CANDIDATES steps by the
// smallest fine residual norm; the choice is made on the device (graph-safe).
int line_search_correction(GlideLevel* L, GlideLevel* C, const GlideSolverConfig* c, void* s) {
    static const double alphas[GLIDE_LS_CANDIDATES] = {1.0, 0.5, 0.25, 0.0};  // same order as ls_pick_k
    LevelView w = view(L), wc = view(C);
    const int64_t ntb = w.ntot * w.nb;
    TRY(glide_prolong(w.dt, 0, 1, 0, wc.u(C->z), w.u(L->z), C->a.ny, C->a.nx, C->a.nb, s));
    TRY(glide_prolong(w.dt, 1, 1, 0, wc.v(C->z), w.v(L->z), C->a.ny, C->a.nx, C->a.nb, s));
    if (c->smooth_H_correction != 2)
        TRY(glide_prolong(w.dt, 2, c->smooth_H_correction, 0, wc.H(C->z), w.H(L->z), C->a.ny, C->a.nx, C->a.nb, s));
    else
        TRY(glide_fill(w.dt, w.H(L->z), 0.0, w.nc * w.nb, s));
    TRY(glide_lincomb(w.dt, L->ls_tmp, L->U, 1.0, nullptr, 0.0, ntb, s));   // U_pre
    for (int j = 0; j < GLIDE_LS_CANDIDATES; j++) {
        TRY(glide_lincomb(w.dt, L->U, L->ls_tmp, 1.0, L->z, alphas[j], ntb, s));
        TRY(glide_residual(&L->a, w.u(L->f), w.v(L->f), w.H(L->f), w.u(L->r), w.v(L->r), w.H(L->r), s));
        TRY(glide_norms(w.dt, L->ls_norms + 3 * j, L->norm_parts, w.u(L->r), w.v(L->r), w.H(L->r), L->a.H,
                        L->a.gamma, w.nu * w.nb, w.nv * w.nb, w.nc * w.nb, s));
    }
    double* a_dev = L->ls_norms + 3 * GLIDE_LS_CANDIDATES;
    TRY(launch_ls_pick(a_dev, L->ls_norms, GLIDE_LS_CANDIDATES, S(s)));
    return (w.dt == GLIDE_F32 ? launch_axpy_dev<float> : launch_axpy_dev<double>)(L->U, L->ls_tmp, a_dev, L->z, ntb,
                                                                                   S(s));
}

int fascd(GlideLevel* lv, int n, int k, bool finest, const GlideSolverConfig* c, void* s) {
    GlideLevel* L = &lv[k];
    LevelView w = view(L);
    const int64_t ncb = w.nc * w.nb, ntb = w.ntot * w.nb;
    if (finest) {
        TRY(glide_lincomb(w.dt, L->w, L->U, 1.0, nullptr, 0.0, ntb, s));                        // w = U
        TRY(glide_lincomb(w.dt, L->chi, L->a.gamma, 1.0, L->a.H, -1.0, ncb, s));              // chi = gamma - H
    }
    if (k == n - 1) {
        TRY(gamma_from(L, L->chi, s));
        TRY(vanka(L, c->n_coarse, c, false, s));
        return fill_gamma(L, c->thklim, s);
    }
    GlideLevel* C = &lv[k + 1];
    LevelView wc = view(C);
    // chi_c = maxpool(chi); gamma = w_H + (inject(-chi_c) + chi)   (solver.py:101-108)
    TRY((wc.dt == GLIDE_F32 ? launch_constraint_down<float> : launch_constraint_down<double>)(
        C->chi, (void*)L->a.gamma, L->chi, w.H(L->w), C->a.ny, C->a.nx, C->a.nb, (cudaStream_t)s));
    TRY(vanka(L, c->n_smooth, c, false, s));
    TRY(fill_gamma(L, c->thklim, s));
    // restrict the state, child.w = child.U   (solver.py:113-117)
    TRY(restrict3(L, C, L->U, C->U, s));
    TRY(glide_lincomb(wc.dt, C->w, C->U, 1.0, nullptr, 0.0, wc.ntot * wc.nb, s));
    // child.f = F_c(R U) - R r   (solver.py:120-125)
    TRY(glide_residual(&L->a, w.u(L->f), w.v(L->f), w.H(L->f), w.u(L->r), w.v(L->r), w.H(L->r), s));
    TRY(restrict3(L, C, L->r, C->r, s));
    TRY(glide_residual(&C->a, wc.u(C->r), wc.v(C->r), wc.H(C->r), wc.u(C->f), wc.v(C->f), wc.H(C->f), s));
    TRY(fascd(lv, n, k + 1, false, c, s));
    // U += P(U_c - w_c): bilinear for u and v, injection for H   (solver.py:131-140)
    TRY(glide_lincomb(wc.dt, C->z, C->U, 1.0, C->w, -1.0, wc.ntot * wc.nb, s));
    if (finest && c->coarse_line_search && L->ls_tmp && L->ls_norms && L->norm_parts) {
        TRY(line_search_correction(L, C, c, s));
    } else {
        TRY(glide_prolong(w.dt, 0, 1, 1, wc.u(C->z), w.u(L->U), C->a.ny, C->a.nx, C->a.nb, s));
        TRY(glide_prolong(w.dt, 1, 1, 1, wc.v(C->z), w.v(L->U), C->a.ny, C->a.nx, C->a.nb, s));
        if (c->smooth_H_correction != 2)  // 2: velocity-only coarse correction
            TRY(glide_prolong(w.dt, 2, c->smooth_H_correction, 1, wc.H(C->z), w.H(L->U), C->a.ny, C->a.nx,
                              C->a.nb, s));
    }
    // post-smoothing and local error-driven smoothing   (solver.py:143-157)
    TRY(gamma_from(L, L->chi, s));
    TRY(vanka(L, c->n_smooth, c, false, s));
    for (int it = 0; it < c->n_local_outer; it++) {
        TRY(glide_residual(&L->a, w.u(L->f), w.v(L->f), w.H(L->f), w.u(L->r), w.v(L->r), w.H(L->r), s));
        TRY(glide_error_mask(&L->a, w.u(L->r), w.v(L->r), w.H(L->r), c->err_threshold, L->err_mask, L->flags,
                             L->any_active, s));
        TRY(vanka(L, c->n_local, c, true, s));
    }
    return fill_gamma(L, c->thklim, s);
}

int mask_on(GlideLevel* L, const GlideSolverConfig* c, void* s) {
    LevelView w = view(L);
    const double tol = c->adj_active_tol > 0.0 ? c->adj_active_tol : 0.1;   // glide/grid.py:332-334
    return glide_mask_le(w.dt, (void*)L->a.mask, L->a.H, L->a.gamma, tol, w.nc * w.nb, s);
}
int mask_off(GlideLevel* L, void* s) {
    LevelView w = view(L);
    return glide_fill(w.dt, (void*)L->a.mask, 0.0, w.nc * w.nb, s);
}

// r_adj = f_adj - VJP(lambda) with the current mask
int adj_residual(GlideLevel* L, int exact, void* s) {
    LevelView w = view(L);
    return glide_vjp(&L->a, w.u(L->lam), w.v(L->lam), w.H(L->lam), w.u(L->f_adj), w.v(L->f_adj), w.H(L->f_adj),
                     w.u(L->r_adj), w.v(L->r_adj), w.H(L->r_adj), exact, s);
}

int vanka_adj(GlideLevel* L, int n_iter, double omega, int exact, void* s) {
    LevelView w = view(L);
    for (int it = 0; it < n_iter; it++) {
        for (int color = 0; color < 2; color++) {
            TRY(adj_residual(L, exact, s));
            TRY(glide_vanka_adjoint(&L->a, w.u(L->lam), w.v(L->lam), w.H(L->lam), w.u(L->r_adj), w.v(L->r_adj),
                                    w.H(L->r_adj), color, omega, s));
        }
    }
    return 0;
}

int restrict_params(GlideLevel* L, GlideLevel* C, void* s) {
    LevelView w = view(L);
    const int nyc = C->a.ny, nxc = C->a.nx, nb = C->a.nb;
    TRY(glide_restrict(w.dt, 2, 0, L->a.bed, (void*)C->a.bed, nyc, nxc, nb, s));
    TRY(glide_restrict(w.dt, 2, 0, L->a.B, (void*)C->a.B, nyc, nxc, nb, s));
    TRY(glide_restrict(w.dt, 2, 0, L->a.beta, (void*)C->a.beta, nyc, nxc, nb, s));
    if (L->H_prev && C->H_prev) TRY(glide_restrict(w.dt, 2, 0, L->H_prev, C->H_prev, nyc, nxc, nb, s));
    if (L->smb && C->smb) TRY(glide_restrict(w.dt, 2, 0, L->smb, C->smb, nyc, nxc, nb, s));
    return 0;
}

int adjoint(GlideLevel* lv, int n, int k, const GlideSolverConfig* c, void* s) {
    GlideLevel* L = &lv[k];
    LevelView w = view(L);
    const int ex = c->exact_adjoint;
    if (k == n - 1) {
        TRY(mask_on(L, c, s));
        TRY(vanka_adj(L, c->adj_coarse, c->adj_omega, ex, s));
        return mask_off(L, s);
    }
    GlideLevel* C = &lv[k + 1];
    LevelView wc = view(C);
    TRY(mask_on(L, c, s));
    TRY(vanka_adj(L, c->adj_smooth, c->adj_omega, ex, s));
    TRY(mask_off(L, s));
    TRY(adj_residual(L, ex, s));                               // solver.py:187-189 (mask = 0)
    TRY(restrict_params(L, C, s));                             // solver.py:193
    TRY(restrict3(L, C, L->r_adj, C->f_adj, s));               // solver.py:196-199
    TRY(glide_fill(wc.dt, C->lam, 0.0, wc.ntot * wc.nb, s));   // solver.py:200
    TRY(adjoint(lv, n, k + 1, c, s));
    TRY(glide_prolong(w.dt, 0, 1, 1, wc.u(C->lam), w.u(L->lam), C->a.ny, C->a.nx, C->a.nb, s));
    TRY(glide_prolong(w.dt, 1, 1, 1, wc.v(C->lam), w.v(L->lam), C->a.ny, C->a.nx, C->a.nb, s));
    TRY(glide_prolong(w.dt, 2, 1, 1, wc.H(C->lam), w.H(L->lam), C->a.ny, C->a.nx, C->a.nb, s));
    TRY(mask_on(L, c, s));
    TRY(vanka_adj(L, c->adj_smooth, c->adj_omega, ex, s));
    return mask_off(L, s);
}

// --- linear multigrid of the Newton-Krylov finishing solver -------------------
int lin_ready(GlideLevel* lv, int n) {
    for (int k = 0; k < n; k++)
        if (!lv[k].lu || !lv[k].lin_rhs || !lv[k].lin_rho || !lv[k].lin_d || !lv[k].r_raw || !lv[k].scratch)
            return GLIDE_E_NULL;
    return 0;
}

int linear_setup(GlideLevel* lv, int n, const GlideSolverConfig* c, void* s) {
    TRY(fill_gamma(&lv[0], c->thklim, s));
    for (int k = 1; k < n; k++) {
        GlideLevel *F = &lv[k - 1], *L = &lv[k];
        LevelView w = view(L);
        TRY(restrict3(F, L, F->U, L->U, s));
        TRY(restrict3(F, L, F->r_raw, L->r_raw, s));
        TRY(fill_gamma(L, c->thklim, s));
        TRY(glide_active_mask(&L->a, w.H(L->r_raw), (void*)L->a.mask, s));
    }
    for (int k = 0; k < n; k++) TRY(glide_vanka_lu_masked(&lv[k].a, lv[k].lu, c->lin_shift, s));
    return 0;
}

// rho = rhs + J d on level L
int lin_residual(GlideLevel* L, void* s) {
    LevelView w = view(L);
    return glide_jvp_add(&L->a, w.u(L->lin_d), w.v(L->lin_d), w.H(L->lin_d), w.u(L->lin_rhs), w.v(L->lin_rhs),
                         w.H(L->lin_rhs), w.u(L->lin_rho), w.v(L->lin_rho), w.H(L->lin_rho), s);
}

int lin_sweeps(GlideLevel* L, int n_sweeps, bool from_zero, const GlideSolverConfig* c, void* s) {
    LevelView w = view(L);
    for (int it = 0; it < n_sweeps; it++) {
        void* rho = L->lin_rho;
        if (it == 0 && from_zero) rho = L->lin_rhs;   // d = 0: rho = rhs
        else TRY(lin_residual(L, s));
        TRY(glide_vanka_linear(&L->a, w.u(rho), w.v(rho), w.H(rho), L->lu, w.u(L->lin_d), w.v(L->lin_d),
                               w.H(L->lin_d), c->lin_omega, L->scratch, s));
    }
    return 0;
}

int lin_vcycle(GlideLevel* lv, int n, int k, const GlideSolverConfig* c, void* s) {
    GlideLevel* L = &lv[k];
    LevelView w = view(L);
    TRY(glide_fill(w.dt, L->lin_d, 0.0, w.ntot * w.nb, s));
    if (k == n - 1) return lin_sweeps(L, c->lin_coarse, true, c, s);
    TRY(lin_sweeps(L, c->lin_pre, true, c, s));
    GlideLevel* C = &lv[k + 1];
    LevelView wc = view(C);
    TRY(lin_residual(L, s));
    TRY(restrict3(L, C, L->lin_rho, C->lin_rhs, s));
    TRY(lin_vcycle(lv, n, k + 1, c, s));
    TRY(glide_prolong(w.dt, 0, 1, 1, wc.u(C->lin_d), w.u(L->lin_d), C->a.ny, C->a.nx, C->a.nb, s));
    TRY(glide_prolong(w.dt, 1, 1, 1, wc.v(C->lin_d), w.v(L->lin_d), C->a.ny, C->a.nx, C->a.nb, s));
    TRY(glide_prolong(w.dt, 2, 1, 1, wc.H(C->lin_d), w.H(L->lin_d), C->a.ny, C->a.nx, C->a.nb, s));
    return lin_sweeps(L, c->lin_post, false, c, s);
}

int check_levels(GlideLevel* lv, int n) {
    if (!lv || n < 1) return GLIDE_E_NULL;
    for (int k = 0; k < n; k++) {
        int e = check_level(&lv[k].a);
        if (e) return e;
        if (lv[k].a.dtype != lv[0].a.dtype) return GLIDE_E_DTYPE;
        if (k > 0 && (lv[k].a.ny * 2 != lv[k - 1].a.ny || lv[k].a.nx * 2 != lv[k - 1].a.nx)) return GLIDE_E_SHAPE;
    }
    return 0;
}

struct GraphHandle {
    cudaGraph_t g;
    cudaGraphExec_t e;
};

}  // namespace

extern "C" {

int glide_fascd_vcycle(GlideLevel* levels, int n_levels, int k0, int finest, const GlideSolverConfig* cfg,
                       void* stream) {
    int e = check_levels(levels, n_levels);
    if (e) return e;
    if (!cfg || k0 < 0 || k0 >= n_levels) return GLIDE_E_SHAPE;
    return fascd(levels, n_levels, k0, finest != 0, cfg, stream);
}

int glide_adjoint_vcycle(GlideLevel* levels, int n_levels, int k0, const GlideSolverConfig* cfg, void* stream) {
    int e = check_levels(levels, n_levels);
    if (e) return e;
    if (!cfg || k0 < 0 || k0 >= n_levels) return GLIDE_E_SHAPE;
    return adjoint(levels, n_levels, k0, cfg, stream);
}

int glide_restrict_parameters(GlideLevel* levels, int n_levels, int k0, void* stream) {
    int e = check_levels(levels, n_levels);
    if (e) return e;
    for (int k = k0; k + 1 < n_levels; k++) TRY(restrict_params(&levels[k], &levels[k + 1], stream));
    return 0;
}

int glide_linear_setup(GlideLevel* levels, int n_levels, const GlideSolverConfig* cfg, void* stream) {
    int e = check_levels(levels, n_levels);
    if (e) return e;
    if (!cfg) return GLIDE_E_NULL;
    if ((e = lin_ready(levels, n_levels))) return e;
    return linear_setup(levels, n_levels, cfg, stream);
}

int glide_linear_vcycle(GlideLevel* levels, int n_levels, const GlideSolverConfig* cfg, void* stream) {
    int e = check_levels(levels, n_levels);
    if (e) return e;
    if (!cfg) return GLIDE_E_NULL;
    if ((e = lin_ready(levels, n_levels))) return e;
    if (cfg->lin_pre < 0 || cfg->lin_post < 0 || cfg->lin_coarse < 1) return GLIDE_E_SHAPE;
    return lin_vcycle(levels, n_levels, 0, cfg, stream);
}

int glide_graph_create(GlideLevel* levels, int n_levels, const GlideSolverConfig* cfg, int kind, void** graph_out) {
    int e = check_levels(levels, n_levels);
    if (e) return e;
    if (!cfg || !graph_out) return GLIDE_E_NULL;
    if (kind < 0 || kind > 2) return GLIDE_E_SHAPE;
    if (kind == 2 && ((e = lin_ready(levels, n_levels)) || cfg->lin_coarse < 1)) return e ? e : GLIDE_E_SHAPE;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return GLIDE_E_GRAPH;
    GraphHandle* h = new GraphHandle();
    int rc = 0;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = GLIDE_E_GRAPH;
    if (!rc) {
        rc = kind == 0   ? fascd(levels, n_levels, 0, true, cfg, s)
             : kind == 1 ? adjoint(levels, n_levels, 0, cfg, s)
                         : lin_vcycle(levels, n_levels, 0, cfg, s);
        cudaError_t ce = cudaStreamEndCapture(s, &h->g);
        if (!rc && ce != cudaSuccess) rc = GLIDE_E_GRAPH;
    }
    if (!rc && cudaGraphInstantiate(&h->e, h->g, 0) != cudaSuccess) rc = GLIDE_E_GRAPH;
    cudaStreamDestroy(s);
    if (rc) {
        delete h;
        return rc;
    }
    *graph_out = h;
    return 0;
}

int glide_graph_launch(void* graph, void* stream) {
    if (!graph) return GLIDE_E_NULL;
    GraphHandle* h = (GraphHandle*)graph;
    return (int)cudaGraphLaunch(h->e, S(stream));
}

int glide_graph_destroy(void* graph) {
    if (!graph) return GLIDE_E_NULL;
    GraphHandle* h = (GraphHandle*)graph;
    cudaGraphExecDestroy(h->e);
    cudaGraphDestroy(h->g);
    delete h;
    return 0;
}

}  // extern "C"
