// Host launchers for the reference's transfer kernels (glide/cuda/utility.cu),
// with the 1-D 256-thread launch of glide/kernels.py:90-236 (test infrastructure).
#include "utility.cu"

#define L1D(n) dim3(((n) + 255) / 256), dim3(256), 0, (cudaStream_t)stream

extern "C" int ref_transfer(int op, const float* src, float* dst, int n_a, int n_b, void* stream) {
    // op: 0 restrict_u, 1 restrict_v, 2 restrict_cell_centered, 3 restrict_max_pool (n_a,n_b = coarse ny,nx)
    //     4 prolongate_u, 5 prolongate_v, 6 prolongate_cell_centered,
    //     7 prolongate_u_smooth, 8 prolongate_v_smooth, 9 prolongate_H_smooth (n_a,n_b = fine ny,nx)
    const int a = n_a, b = n_b;
    switch (op) {
        case 0: restrict_u<<<L1D(a * (b + 1))>>>(src, dst, a, b); break;
        case 1: restrict_v<<<L1D((a + 1) * b)>>>(src, dst, a, b); break;
        case 2: restrict_cell_centered<<<L1D(a * b)>>>(src, dst, a, b); break;
        case 3: restrict_max_pool<<<L1D(a * b)>>>(src, dst, a, b); break;
        case 4: prolongate_u<<<L1D(a * (b + 1))>>>(src, dst, a, b); break;
        case 5: prolongate_v<<<L1D((a + 1) * b)>>>(src, dst, a, b); break;
        case 6: prolongate_cell_centered<<<L1D(a * b)>>>(src, dst, a, b); break;
        case 7: prolongate_u_smooth<<<L1D(a * (b + 1))>>>(src, dst, a, b); break;
        case 8: prolongate_v_smooth<<<L1D((a + 1) * b)>>>(src, dst, a, b); break;
        case 9: prolongate_H_smooth<<<L1D(a * b)>>>(src, dst, a, b); break;
        default: return -2;
    }
    return (int)cudaGetLastError();
}
