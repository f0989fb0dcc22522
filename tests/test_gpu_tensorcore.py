"""tcgen05 BF16 GEMM and the convolution data kernels vs a plain PyTorch FP32
reference of the same op.

Tolerance: the GEMM consumes BF16 inputs exactly and accumulates in FP32, so
it is compared with an FP32 product of the same BF16 values: max abs error
<= 1e-3 * (max |ref| + 1) (FP32 summation-order differences only).  im2col,
col2im and transposes are data movement: exact.
"""
import ctypes as C

import pytest
import torch

pytestmark = pytest.mark.gpu


def _lib():
    from glide_b200 import _native as N
    lib = N.load()
    lib.glide_gemm_bf16.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    lib.glide_im2col3_bf16.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 5 + [C.c_void_p]
    lib.glide_col2im3_f32.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 5 + [C.c_void_p]
    lib.glide_transpose_bf16.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    return lib


def gemm(A, B, bias=None, relu=False, out_mode=0, C_out=None):
    lib = _lib()
    M, K = A.shape
    N = B.shape[0]
    if C_out is None:
        C_out = torch.zeros((M, N), dtype=torch.bfloat16 if out_mode == 1 else torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.glide_gemm_bf16(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), C_out.data_ptr(), C_out.stride(0),
                             M, N, K, None if bias is None else bias.data_ptr(), int(relu), out_mode, err.data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C_out


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 128, 288), (1000, 96, 72), (77, 32, 16), (640, 256, 576)])
def test_gemm_matches_fp32(M, N, K):
    torch.manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda").bfloat16()
    B = torch.randn(N, K, device="cuda").bfloat16()
    ref = A.float() @ B.float().T
    out = gemm(A, B)
    assert (out - ref).abs().max().item() <= 1e-3 * (ref.abs().max().item() + 1)


def test_gemm_epilogue_bias_relu_bf16_and_accumulate():
    torch.manual_seed(1)
    A = torch.randn(300, 144, device="cuda").bfloat16()
    B = torch.randn(64, 144, device="cuda").bfloat16()
    bias = torch.randn(64, device="cuda")
    ref = torch.relu(A.float() @ B.float().T + bias)
    out = gemm(A, B, bias=bias, relu=True, out_mode=1)
    assert (out.float() - ref).abs().max().item() <= 1e-2 * (ref.abs().max().item() + 1)
    acc = torch.ones(300, 64, device="cuda")
    gemm(A, B, out_mode=2, C_out=acc)
    assert (acc - (1 + A.float() @ B.float().T)).abs().max().item() <= 1e-3 * (ref.abs().max().item() + 1)


def test_im2col_col2im_conv_adjoint():
    lib = _lib()
    torch.manual_seed(2)
    Bn, H, W, Cc = 2, 9, 13, 8
    Kp = 9 * Cc
    x = torch.randn(Bn, H, W, Cc, device="cuda").bfloat16()
    col = torch.empty(Bn * H * W, Kp, dtype=torch.bfloat16, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.glide_im2col3_bf16(x.data_ptr(), col.data_ptr(), Bn, H, W, Cc, Kp, s) == 0
    w = torch.randn(5, Cc, 3, 3, device="cuda")
    # conv via im2col equals torch conv2d (NCHW) on the same bf16 values
    wk = w.permute(0, 2, 3, 1).reshape(5, Kp)  # (co, ky, kx, ci)
    y = (col.float() @ wk.T).reshape(Bn, H, W, 5).permute(0, 3, 1, 2)
    # CPU FP32 reference (CUDA conv2d would use TF32)
    ref = torch.nn.functional.conv2d(x.float().permute(0, 3, 1, 2).cpu(), w.cpu(), padding=1)
    assert (y.cpu() - ref).abs().max().item() < 1e-3
    # col2im is the adjoint of im2col: <col(x), d> == <x, col2im(d)>
    d = torch.randn(Bn * H * W, Kp, device="cuda")
    dx = torch.empty(Bn, H, W, Cc, device="cuda")
    assert lib.glide_col2im3_f32(d.data_ptr(), dx.data_ptr(), Bn, H, W, Cc, Kp, s) == 0
    torch.cuda.synchronize()
    a = (col.float() * d).sum().item()
    b = (x.float() * dx).sum().item()
    assert abs(a - b) <= 1e-4 * abs(a)


def test_transpose():
    lib = _lib()
    x = torch.randn(70, 45, device="cuda").bfloat16()
    y = torch.empty(45, 70, dtype=torch.bfloat16, device="cuda")
    assert lib.glide_transpose_bf16(x.data_ptr(), y.data_ptr(), 70, 45, torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert torch.equal(y, x.T)


@pytest.mark.parametrize("C_in,C_out,out_mode", [(8, 32, 1), (32, 64, 1), (96, 32, 0), (64, 128, 1)])
def test_implicit_conv3x3_equals_im2col_gemm(C_in, C_out, out_mode):
    """glide_conv3x3_bf16 (im2col gathered while staging each tile) against
    glide_im2col3_bf16 + glide_gemm_bf16 on the same inputs: the staged tiles
    are the same, so the results are bit-identical (ragged M and N edges,
    zero padding at the image border, bias and ReLU in the epilogue)."""
    from glide_b200.guess import conv3x3, gemm as lib_gemm, im2col3
    g = torch.Generator(device="cuda").manual_seed(C_in + C_out)
    x = torch.randn(2, 37, 45, C_in, generator=g, device="cuda").to(torch.bfloat16)
    Wb = (torch.randn(C_out, 9 * C_in, generator=g, device="cuda") * 0.1).to(torch.bfloat16)
    bias = torch.randn(C_out, generator=g, device="cuda")
    dt = torch.bfloat16 if out_mode == 1 else torch.float32
    a = torch.empty((2 * 37 * 45, C_out), dtype=dt, device="cuda")
    b = torch.empty_like(a)
    lib_gemm(im2col3(x), Wb, a, bias=bias, relu=True, out_mode=out_mode)
    conv3x3(x, Wb, b, bias=bias, relu=True, out_mode=out_mode)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("N", [24, 64, 96, 200])
def test_pipelined_and_single_stage_gemm_agree(N):
    """Aligned operands run the cp.async-pipelined kernel (N tile 32, 64 or
    128 after the output width); an A with a row pitch that is not a multiple
    of 8 elements runs the single-stage kernel.  Both accumulate the same BF16
    products in FP32 chunk by chunk: results agree to FP32 rounding, and both
    match the FP32 product."""
    torch.manual_seed(N)
    M, K = 300, 136
    A = torch.randn(M, K, device="cuda").bfloat16()
    B = torch.randn(N, K, device="cuda").bfloat16()
    A_pad = torch.zeros(M, K + 4, device="cuda").bfloat16()
    A_pad[:, :K] = A
    bias = torch.randn(N, device="cuda")
    p = gemm(A, B, bias=bias, relu=True, out_mode=0)
    s = gemm(A_pad[:, :K], B, bias=bias, relu=True, out_mode=0)
    ref = torch.relu(A.float() @ B.float().T + bias)
    assert (p - s).abs().max().item() <= 1e-5 * (ref.abs().max().item() + 1)
    assert (p - ref).abs().max().item() <= 1e-3 * (ref.abs().max().item() + 1)
