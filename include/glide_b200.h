/*
 * glide_b200 C ABI: the SSA forward/adjoint hot path of GLIDE on one B200.
 *
 * Plain C types only (device pointers, sizes, a cudaStream_t passed as
 * void*).  Every function returns 0 on success, a negative GLIDE_E_* code for
 * invalid arguments, or a positive CUDA error code from the launch.  Nothing
 * here allocates device memory; the caller owns every buffer.
 *
 * Grid layout (MAC staggered, glide/grid.py:1-8 of the reference):
 *   u  (ny, nx+1) on vertical faces, v (ny+1, nx) on horizontal faces,
 *   H and cell parameters (ny, nx); a batch of nb problems is stored
 *   back to back (problem b at offset b * field_size).
 * dtype: GLIDE_F32 or GLIDE_F64 for every floating-point buffer of a call.
 *
 * Reference interfaces replaced (paths inside glide-ism/glide):
 *   glide_residual       <- compute_residual  glide/cuda/residuals.cu:6-24
 *   glide_jvp            <- compute_jvp       glide/cuda/residuals.cu:299-317
 *   glide_vjp            <- compute_vjp       glide/cuda/residuals.cu:586-604
 *   glide_grad_beta      <- compute_grad_beta glide/cuda/grad.cu:1-17
 *   glide_vanka_sweeps   <- vanka_smooth / vanka_smooth_local glide/cuda/vanka.cu:3-23,844-864
 *                           + Grid.vanka_sweep(_local) glide/grid.py:305-317
 *   glide_error_mask     <- error indicator of glide/solver.py:147-154
 *   glide_vanka_adjoint  <- vanka_smooth_adjoint glide/cuda/vanka.cu:441-464
 *   glide_restrict / glide_prolong <- restrict_* / prolongate_* glide/cuda/utility.cu:1-337,
 *                           wrappers glide/kernels.py:90-236
 *   glide_fascd_vcycle   <- fascd_vcycle   glide/solver.py:71-157
 *   glide_adjoint_vcycle <- adjoint_vcycle glide/solver.py:160-220
 *   GlidePhysicsParams   <- PhysicsParams  glide/cuda/common.cu:240-247 (same fields, double precision)
 */
#ifndef GLIDE_B200_H
#define GLIDE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GLIDE_F32 0
#define GLIDE_F64 1

#define GLIDE_OK 0
#define GLIDE_E_DTYPE (-1)
#define GLIDE_E_SHAPE (-2)
#define GLIDE_E_NULL (-3)
#define GLIDE_E_GRAPH (-4)
#define GLIDE_E_TOO_LARGE (-5)  /* a field of one problem reaches 2^31 elements, or a fixed buffer is too small */

/* Fraction of each local Newton step the reference's Vanka smoother takes
 * (relaxation_factor, glide/cuda/vanka.cu:416). */
#define GLIDE_REF_NEWTON_STEP 0.25

typedef struct GlidePhysicsParams {
    double n;             /* Glen exponent */
    double eps_reg;       /* strain-rate regularisation */
    double water_drag;    /* drag under floating ice */
    double calving_rate;
    double gl_sigmoid_c;  /* grounding-line sigmoid sharpness */
    int gl_derivatives;   /* include dH terms through the grounding sigmoid */
} GlidePhysicsParams;

/* One level (or a batch of equal-sized levels) and its state/parameters. */
typedef struct GlideLevelArgs {
    int ny, nx, nb, dtype;
    double dx, dt;
    GlidePhysicsParams params;
    const void *u, *v, *H;               /* state; written by the smoothers */
    const void *bed, *B, *beta;          /* cell parameters */
    const void *mask, *gamma;            /* active-set mask and thickness limit, cells */
} GlideLevelArgs;

/* r = F(U) - f with the active-set row (1-m) r_H + m (H - gamma). */
int glide_residual(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, void* r_u, void* r_v,
                   void* r_H, void* stream);
/* J(U) d. */
int glide_jvp(const GlideLevelArgs* a, const void* d_u, const void* d_v, const void* d_H, void* j_u, void* j_v,
              void* j_H, void* stream);
/* out = base + J(U) d in one pass: the linear residual r + J d of a defect
 * correction.  No counterpart in the reference (its defect correction is
 * not linearised); same J as glide_jvp.  out must not overlap base or d
 * (GLIDE_E_SHAPE when a pointer pair is equal). */
int glide_jvp_add(const GlideLevelArgs* a, const void* d_u, const void* d_v, const void* d_H, const void* base_u,
                  const void* base_v, const void* base_H, void* out_u, void* out_v, void* out_H, void* stream);
/* lambda^T J(U); with f_u/f_v/f_H non-null writes f - lambda^T J instead.
 * exact_boundary = 0 reproduces the reference's boundary handling. */
int glide_vjp(const GlideLevelArgs* a, const void* l_u, const void* l_v, const void* l_H, const void* f_u,
              const void* f_v, const void* f_H, void* o_u, void* o_v, void* o_H, int exact_boundary, void* stream);
/* grad_beta[c] = sum_faces lambda_face d tau_b / d beta_c (overwrites grad). */
int glide_grad_beta(const GlideLevelArgs* a, const void* l_u, const void* l_v, void* grad, int exact_boundary,
                    void* stream);
/* n_iter Vanka sweeps, each U += omega * delta (u, v, H of a updated in place).
 * shift: diagonal shift of the local Newton matrix (reference: 1.0).
 * flags/any_active non-null: local sweep gated by glide_error_mask's flags.
 * scratch: 5 * ny * nx * nb elements of dtype. */
int glide_vanka_sweeps(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_iter,
                       int n_newton, double omega, double shift, const int* flags, const int* any_active,
                       void* scratch, void* stream);
/* glide_vanka_sweeps with the local Newton step fraction as an argument
 * (0 < newton_step <= 1; the reference fixes it at GLIDE_REF_NEWTON_STEP) and
 * pivoted_lu != 0 solving the local systems with row pivoting (the
 * reference's lu_5x5_solve_pivot, glide/cuda/common.cu:180-233, which its
 * kernels do not call).  Extension, no counterpart in the reference: the
 * tolerance solver's finishing sweeps take full local Newton steps with few
 * iterations. */
int glide_vanka_sweeps_ex(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_iter,
                          int n_newton, double newton_step, double omega, double shift, int pivoted_lu,
                          const int* flags, const int* any_active, void* scratch, void* stream);
/* Same sweeps as glide_vanka_sweeps for callers that cannot allocate device
 * memory (no counterpart in the reference): the scratch lives in a fixed
 * 10 MiB device array inside the library (glide_noalloc_scratch_bytes()),
 * enough for nb*ny*nx <= 262144 cells in FP64 or 524288 in FP32; larger
 * problems return GLIDE_E_TOO_LARGE.  The first call on a device (with that
 * device current) looks up the array's device address and keeps it for that
 * CUDA context; a call in a new context of the device (after
 * cudaDeviceReset) looks it up again.  Make the first call, and the first
 * after a reset, before any stream capture.  All calls share the array, so
 * calls that overlap on the GPU race and must be ordered by the caller.
 * Allocates nothing. */
int glide_vanka_sweeps_noalloc(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_iter,
                               int n_newton, double omega, double shift, const int* flags, const int* any_active,
                               void* stream);
size_t glide_noalloc_scratch_bytes(void);
/* Linear Vanka for defect correction (no counterpart in the reference: the
 * tolerance solver's FP32 correction of an FP64 state).  glide_vanka_lu
 * factors every cell's local 5x5 matrix at the state in a (the matrix of the
 * first local Newton iteration of glide_vanka_sweeps with right-hand side
 * f_H in the mass row's active-set test, diagonal shifted by shift) into lu
 * (25 * ny * nx * nb elements).  glide_vanka_linear makes one
 * additive sweep for the correction d of the linear problem r + J d = 0:
 * rho = r + J d is the caller's linear residual; d += omega * (face average
 * of -A^-1 rho), with H + d_H kept >= gamma.  scratch as for the sweeps. */
int glide_vanka_lu(const GlideLevelArgs* a, const void* f_H, void* lu, double shift, void* stream);
int glide_vanka_linear(const GlideLevelArgs* a, const void* rho_u, const void* rho_v, const void* rho_H,
                       const void* lu, void* d_u, void* d_v, void* d_H, double omega, void* scratch, void* stream);
/* Only the per-cell local Newton kernel of a sweep, n_launch times, writing the
 * per-cell deltas into scratch without updating U (profiling and timing). */
int glide_vanka_cells(const GlideLevelArgs* a, const void* f_u, const void* f_v, const void* f_H, int n_launch,
                      int n_newton, double shift, const int* flags, const int* any_active, void* scratch,
                      void* stream);
/* err_mask = (|r_u|+|r_u|+|r_v|+|r_v|+|FB(r_H,H-gamma)| > threshold); if flags
 * is non-null also the per-reference-block flags ((ny/14+1)*(nx/14+1)*nb ints)
 * and any_active (nb ints). */
int glide_error_mask(const GlideLevelArgs* a, const void* r_u, const void* r_v, const void* r_H, double threshold,
                     void* err_mask, int* flags, int* any_active, void* stream);
/* Block flags from an existing error mask. */
int glide_tile_flags(const GlideLevelArgs* a, const void* err_mask, int* flags, int* any_active, void* stream);
/* One colour of the red-black adjoint Vanka; lambda updated in place. */
int glide_vanka_adjoint(const GlideLevelArgs* a, void* l_u, void* l_v, void* l_H, const void* ra_u, const void* ra_v,
                        const void* ra_H, int color, double omega, void* stream);

/* Transfers.  field: 0 = u faces, 1 = v faces, 2 = cells; sizes of the coarse grid. */
int glide_restrict(int dtype, int field, int use_max, const void* fine, void* coarse, int nyc, int nxc, int nb,
                   void* stream);
int glide_prolong(int dtype, int field, int smooth, int add, const void* coarse, void* fine, int nyc, int nxc, int nb,
                  void* stream);
/* out = a*x + b*y (y may be null), n elements. */
int glide_lincomb(int dtype, void* out, const void* x, double a, const void* y, double b, int64_t n, void* stream);
int glide_fill(int dtype, void* out, double val, int64_t n, void* stream);
/* mask = H <= gamma + tol */
int glide_mask_le(int dtype, void* mask, const void* H, const void* gamma, double tol, int64_t n, void* stream);
/* Convert between f32 and f64 buffers (out dtype = dst_dtype); out = x (+ add_to_out ? out : 0). */
int glide_convert(int dst_dtype, void* out, const void* x, int64_t n, int accumulate, void* stream);
/* Sums of squares of r_u, r_v, FB(r_H, H-gamma) into out3 (device double[3]);
 * parts: glide_norm_parts(n) * 3 doubles of scratch.  Deterministic. */
int glide_norms(int dtype, double* out3, double* parts, const void* r_u, const void* r_v, const void* r_H,
                const void* H, const void* gamma, int64_t nu, int64_t nv, int64_t nc, void* stream);
int glide_norm_parts(int64_t n);

/* ---- multigrid driver ------------------------------------------------------ */
/* Buffers of one level; U = [u|v|H] monolithic, likewise f, w, r, z, lam,
 * f_adj, r_adj.  a.u/a.v/a.H must point into U. */
typedef struct GlideLevel {
    GlideLevelArgs a;
    void *U, *f, *w, *r, *z;
    void *chi, *err_mask;
    void *lam, *f_adj, *r_adj;
    void *H_prev, *smb;
    void* scratch;          /* 5 * nc * nb */
    int* flags;             /* (ny/14+1) * (nx/14+1) * nb */
    int* any_active;        /* nb */
    /* coarse-correction line search (finest level; may be null when off) */
    void* ls_tmp;           /* one state vector (like U) */
    double* ls_norms;       /* 3 * GLIDE_LS_CANDIDATES + 1 doubles */
    double* norm_parts;     /* 3 * glide_norm_parts(max(nu, nc) * nb) doubles */
    /* linear multigrid of the Newton-Krylov finishing solver (may be null when
       glide_linear_setup / glide_linear_vcycle are not used) */
    void* lu;               /* 25 * nc * nb: local Vanka factors at the level's state */
    void* lin_rhs;          /* like U: right-hand side g of J d = -g */
    void* lin_rho;          /* like U: linear residual g + J d */
    void* lin_d;            /* like U: correction d */
    void* r_raw;            /* like U: residual at the linearisation state (active-set test) */
} GlideLevel;

/* Step sizes tried by the coarse-correction line search, best first on ties. */
#define GLIDE_LS_CANDIDATES 4

typedef struct GlideSolverConfig {
    double thklim;
    int n_coarse, n_smooth, n_local_outer, n_local, n_newton;
    double omega, shift, err_threshold;
    int adj_coarse, adj_smooth;
    double adj_omega;
    int exact_adjoint;      /* 0: reference VJP boundary handling */
    int smooth_H_correction;/* 0: inject the coarse H correction (reference), 1: bilinear,
                               2: no H correction (velocity-only coarse correction) */
    double newton_step;     /* fraction of each local Newton step taken in the forward sweeps;
                               <= 0 means the reference's GLIDE_REF_NEWTON_STEP */
    int pivoted_lu;         /* 1: local 5x5 systems of the forward sweeps solved with row pivoting */
    int coarse_line_search; /* 1: on the finest level, U = U_pre + a * P(U_c - w_c) with a in
                               {1, 1/2, 1/4, 0} minimising the residual norm (chosen on the
                               device); 0: a = 1 (reference) */
    /* linear V-cycle of the Newton-Krylov finishing solver (glide_linear_vcycle) */
    int lin_pre, lin_post;  /* linear Vanka sweeps before / after the coarse correction */
    int lin_coarse;         /* linear sweeps on the coarsest level */
    double lin_omega;       /* damping of each linear sweep */
    double lin_shift;       /* diagonal shift of the local factors (0: the local Jacobian) */
    /* adjoint active set: cells with H <= gamma + adj_active_tol are identity rows
       of the adjoint system; <= 0 means the reference's 0.1 m (glide/grid.py:332-334) */
    double adj_active_tol;
} GlideSolverConfig;

/* One FASCD V-cycle from level k0 (finest=1 sets w=U, chi=gamma-H first). */
int glide_fascd_vcycle(GlideLevel* levels, int n_levels, int k0, int finest, const GlideSolverConfig* cfg,
                       void* stream);
int glide_adjoint_vcycle(GlideLevel* levels, int n_levels, int k0, const GlideSolverConfig* cfg, void* stream);
/* restrict bed, B, beta, H_prev, smb from every level to its child (glide/solver.py:53-68) */
int glide_restrict_parameters(GlideLevel* levels, int n_levels, int k0, void* stream);

/* Newton-Krylov finishing solver (no counterpart in the reference, which runs
 * a fixed number of FAS V-cycles): a linear multigrid V-cycle for the
 * correction d of J(U) d = -g, with the additive linear Vanka sweep as the
 * smoother on every level and each coarse level linearised at the restricted
 * state.  glide_linear_setup expects level 0's state, mask (the active set),
 * lin_rhs (g) and r_raw (the residual at U) to be set; it restricts the state
 * and r_raw down the hierarchy, sets each coarse level's active set from
 * H - dt r_H <= gamma (gamma = thklim) and factors every level's local
 * matrices (glide_vanka_lu_masked).  glide_linear_vcycle then writes level
 * 0's lin_d from its lin_rhs (graph-capturable, no host synchronisation). */
int glide_linear_setup(GlideLevel* levels, int n_levels, const GlideSolverConfig* cfg, void* stream);
int glide_linear_vcycle(GlideLevel* levels, int n_levels, const GlideSolverConfig* cfg, void* stream);
/* glide_vanka_lu with the active set given by a->mask (1 = the cell's mass
 * row is the constraint H = gamma) instead of the local residual test. */
int glide_vanka_lu_masked(const GlideLevelArgs* a, void* lu, double shift, void* stream);
/* Newton step helpers (no counterpart in the reference).  glide_newton_rhs:
 * from the FP64 residual r (monolithic, faces then cells) of the FP64 level
 * a64, the active set H - dt r_H <= gamma into mask (cells), the right-hand
 * side rhs (r with active rows replaced by H - gamma) and rraw = r, all three
 * in lin_dtype (GLIDE_F32 for the mixed path, GLIDE_F64 for the FP64 path).
 * glide_newton_update: U64 = base64 + alpha * d (d of d_dtype) with H kept
 * >= gamma.  glide_active_mask: mask = (H - dt r_H <= gamma). */
int glide_newton_rhs(const GlideLevelArgs* a64, const void* r64, void* rhs, void* rraw, void* mask, int lin_dtype,
                     void* stream);
int glide_newton_update(const GlideLevelArgs* a64, void* U64, const void* base64, const void* d, int d_dtype,
                        double alpha, void* stream);
int glide_active_mask(const GlideLevelArgs* a, const void* r_H, void* mask, void* stream);
/* out[i] = sum_j V[i*ldv + j] * w[j], i < k <= 32, FP64 accumulation in a fixed
 * order (deterministic); out: k device doubles; parts: glide_dots_parts(n) * k
 * doubles of scratch.  glide_combine: out = beta * out + alpha * sum_i coef[i]
 * V[i] (coef: k device doubles; beta = 0 does not read out).  The Krylov and
 * Anderson steps of the tolerance solver. */
int glide_dots(int dtype, int64_t n, int k, const void* V, int64_t ldv, const void* w, double* out, double* parts,
               void* stream);
int glide_dots_parts(int64_t n);
int glide_combine(int dtype, int64_t n, int k, const void* V, int64_t ldv, const double* coef, double alpha,
                  void* out, double beta, void* stream);

/* CUDA graphs of whole V-cycles.  kind: 0 = FASCD (finest), 1 = adjoint,
 * 2 = linear V-cycle (glide_linear_vcycle).
 * The graph keeps the device pointers it was built with. */
int glide_graph_create(GlideLevel* levels, int n_levels, const GlideSolverConfig* cfg, int kind, void** graph_out);
int glide_graph_launch(void* graph, void* stream);
int glide_graph_destroy(void* graph);

/* ---- fused loss kernels for the inverse problem (glide/physics.py:262-411) -- */
/* Misfit of (u, v) against (u_obs, v_obs) and its gradient in one pass,
 * NaN differences counted as 0; kind 0: mean |d| per component (abs_loss /
 * abs_grad), kind 1: mean sqrt(d^2 + eps) (huber_loss / huber_grad); both
 * gradients divide by nu as the reference's helpers do.  out3 (device
 * double[3]) = {L_u + L_v, sum_u, sum_v}; parts: glide_loss_parts(max(nu, nv))
 * doubles.  Deterministic. */
int glide_misfit(int dtype, int kind, double eps, const void* u, const void* v, const void* u_obs,
                 const void* v_obs, int64_t nu, int64_t nv, void* grad_u, void* grad_v, double* out3, double* parts,
                 void* stream);
/* Tikhonov term 1/2 sum (neighbour differences)^2 of an (ny, nx) field and
 * its gradient (tikhonov_regularization); out1 = device double[1]. */
int glide_tikhonov(int dtype, const void* field, int ny, int nx, void* grad, double* out1, double* parts,
                   void* stream);
int glide_loss_parts(int64_t n);

/* ---- learned initial guess (no counterpart in the reference) -------------- */
/* C[M,N] (+)= A[M,K] * B[N,K]^T on the tcgen05 tensor cores: A, B BF16 row-major
 * with K contiguous (lda, ldb >= K, 16-byte aligned rows for the fast path),
 * FP32 accumulation in TMEM; epilogue + bias[N] (may be null), ReLU if relu;
 * out_mode 0 = store FP32, 1 = store BF16, 2 = add into FP32.  *err (may be
 * null) is set to 1 if a tensor-core wait ran out (the tile is then skipped). */
int glide_gemm_bf16(const void* A, int lda, const void* B, int ldb, void* C, int ldc, int M, int N, int K,
                    const float* bias, int relu, int out_mode, int* err, void* stream);
/* 3x3 "same" convolution as an implicit GEMM on the tcgen05 tensor cores:
 * out[Bn*H*W, N] (+)= im2col(x) * Wt^T with x NHWC BF16 (C a multiple of 8,
 * 16-byte aligned), Wt (N, ldw >= 9C) BF16 with K = (ky*3+kx)*C + c, the
 * im2col gathered while staging each A tile (no col buffer); epilogue and
 * err as glide_gemm_bf16.  Bit-identical to glide_im2col3_bf16 followed by
 * glide_gemm_bf16 with Kp = 9C. */
int glide_conv3x3_bf16(const void* x, int Bn, int H, int W, int C, const void* Wt, int ldw, void* out, int ldc, int N,
                       const float* bias, int relu, int out_mode, int* err, void* stream);
/* im2col of a 3x3 same convolution on NHWC BF16 x (Bn,H,W,C) into col (Bn*H*W, Kp), Kp >= 9C (zero pad). */
int glide_im2col3_bf16(const void* x, void* col, int Bn, int H, int W, int C, int Kp, void* stream);
/* Transpose of im2col (gather form): dx (Bn,H,W,C) FP32 from dcol (Bn*H*W, Kp) FP32. */
int glide_col2im3_f32(const float* dcol, float* dx, int Bn, int H, int W, int C, int Kp, void* stream);
/* dst (Cc x R) = src (R x Cc)^T, BF16. */
int glide_transpose_bf16(const void* src, void* dst, int R, int Cc, void* stream);

/* Kernel launches issued by this library so far in the process (host-side
 * count; launches recorded into a stream capture count once, at capture). */
long long glide_launch_count(void);

/* Library version string. */
const char* glide_version(void);

#ifdef __cplusplus
}
#endif

#endif
