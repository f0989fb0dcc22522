// Host launchers for the reference's own ice kernels (test infrastructure).
//
// The reference sources are compiled from where they lie, in the order the
// reference concatenates them (glide/kernels.py:66-72), with
// --use_fast_math; this file only adds extern "C" host entry points that
// launch them with the reference's configuration: 16x16 blocks, stride 14,
// halo 1, grid (nx/14+1, ny/14+1) (glide/grid.py:182-188).  The parameter
// struct is passed as a device pointer, as in glide/kernels.py:49.
#include "common.cu"
#include "viscosity.cu"
#include "stress.cu"
#include "flux.cu"
#include "residuals.cu"
#include "vanka.cu"
#include "grad.cu"

#define REF_CFG                                    \
    const int stride = 14, halo = 1;               \
    dim3 grid(nx / stride + 1, ny / stride + 1);   \
    dim3 block(16, 16);                            \
    cudaStream_t st = (cudaStream_t)stream;

typedef const float* cf;

extern "C" int ref_compute_residual(float* r_u, float* r_v, float* r_H, cf u, cf v, cf H, cf f_u, cf f_v, cf f_H,
                                    cf bed, cf B, cf beta, cf mask, cf gamma, const void* params, float dx, float dt,
                                    int ny, int nx, void* stream) {
    REF_CFG
    compute_residual<<<grid, block, 0, st>>>(r_u, r_v, r_H, u, v, H, f_u, f_v, f_H, bed, B, beta, mask, gamma,
                                             (const PhysicsParams*)params, dx, dt, ny, nx, stride, halo);
    return (int)cudaGetLastError();
}

extern "C" int ref_compute_jvp(float* j_u, float* j_v, float* j_H, cf u, cf v, cf H, cf d_u, cf d_v, cf d_H, cf bed,
                               cf B, cf beta, cf mask, cf gamma, const void* params, float dx, float dt, int ny, int nx,
                               void* stream) {
    REF_CFG
    compute_jvp<<<grid, block, 0, st>>>(j_u, j_v, j_H, u, v, H, d_u, d_v, d_H, bed, B, beta, mask, gamma,
                                        (const PhysicsParams*)params, dx, dt, ny, nx, stride, halo);
    return (int)cudaGetLastError();
}

// outputs are accumulated with atomicAdd: the caller zero-fills them (glide/grid.py:245)
extern "C" int ref_compute_vjp(float* o_u, float* o_v, float* o_H, cf u, cf v, cf H, cf l_u, cf l_v, cf l_H, cf bed,
                               cf B, cf beta, cf mask, cf gamma, const void* params, float dx, float dt, int ny, int nx,
                               void* stream) {
    REF_CFG
    compute_vjp<<<grid, block, 0, st>>>(o_u, o_v, o_H, u, v, H, l_u, l_v, l_H, bed, B, beta, mask, gamma,
                                        (const PhysicsParams*)params, dx, dt, ny, nx, stride, halo);
    return (int)cudaGetLastError();
}

// delta outputs accumulated with atomicAdd: zero-filled by the caller (glide/grid.py:305-317)
extern "C" int ref_vanka_smooth(float* du, float* dv, float* dH, float* mask, cf u, cf v, cf H, cf f_u, cf f_v,
                                cf f_H, cf bed, cf B, cf beta, cf gamma, const void* params, float dx, float dt, int ny,
                                int nx, int color, int n_newton, float omega, int local, void* stream) {
    REF_CFG
    if (local)
        vanka_smooth_local<<<grid, block, 0, st>>>(du, dv, dH, mask, u, v, H, f_u, f_v, f_H, bed, B, beta, gamma,
                                                   (const PhysicsParams*)params, dx, dt, ny, nx, stride, halo, color,
                                                   n_newton, omega);
    else
        vanka_smooth<<<grid, block, 0, st>>>(du, dv, dH, mask, u, v, H, f_u, f_v, f_H, bed, B, beta, gamma,
                                             (const PhysicsParams*)params, dx, dt, ny, nx, stride, halo, color,
                                             n_newton, omega);
    return (int)cudaGetLastError();
}

extern "C" int ref_vanka_smooth_adjoint(float* lo_u, float* lo_v, float* lo_H, cf l_u, cf l_v, cf l_H, cf mask,
                                        cf ra_u, cf ra_v, cf ra_H, cf u, cf v, cf H, cf bed, cf B, cf beta, cf gamma,
                                        const void* params, float dx, float dt, int ny, int nx, int color, float omega,
                                        void* stream) {
    REF_CFG
    vanka_smooth_adjoint<<<grid, block, 0, st>>>(lo_u, lo_v, lo_H, l_u, l_v, l_H, mask, ra_u, ra_v, ra_H, u, v, H,
                                                 bed, B, beta, gamma, (const PhysicsParams*)params, dx, dt, ny, nx,
                                                 stride, halo, color, omega);
    return (int)cudaGetLastError();
}

// grad accumulated with atomicAdd: zero-filled by the caller (glide/grid.py:341)
extern "C" int ref_compute_grad_beta(float* grad, cf u, cf v, cf H, cf l_u, cf l_v, cf l_H, cf bed, cf B, cf beta,
                                     cf mask, cf gamma, const void* params, float dx, float dt, int ny, int nx,
                                     void* stream) {
    REF_CFG
    compute_grad_beta<<<grid, block, 0, st>>>(grad, u, v, H, l_u, l_v, l_H, bed, B, beta, mask, gamma,
                                              (const PhysicsParams*)params, dx, dt, ny, nx, stride, halo);
    return (int)cudaGetLastError();
}
