"""Learned initial guess: a small U-Net on the B200 tensor cores.

Maps cell fields (H, bed, log beta, B) to cell-centred velocities (u, v),
which are averaged onto the staggered faces and handed to
``IcePhysics.forward(guess=...)``; the plain V-cycle always finishes the
solve and drops the guess if the first cycle does not cut the residual by
``guess_min_reduction``.

Network: 4 resolution levels, 32 base channels (32-64-128-256), two 3x3
conv + ReLU per level, 2x average pooling down, nearest upsampling and skip
concatenation up, a 1x1 head to 2 channels.  Activations are NHWC BF16,
weights are kept in FP32 for the optimiser and cast to BF16 for the
products.  Every convolution runs on the tcgen05 BF16 GEMM with FP32
accumulation in TMEM: in training (forward, data gradient, weight gradient)
as im2col + ``glide_gemm_bf16``, in inference as an implicit GEMM that
gathers the im2col rows while staging each tile (``glide_conv3x3_bf16``);
bias and ReLU are fused into the GEMM epilogue.
Pooling, upsampling, concatenation and the optimiser are element-wise torch
glue.  This part has no counterpart in the reference.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

import torch

from . import _native as N

DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "guess_weights.pt"
VEL_SCALE = 100.0          # m/a
IN_CH = 8                  # 4 physical inputs zero-padded to 8 channels (16-byte rows)


def _lib():
    lib = N.load()
    if not getattr(lib, "_guess_sigs", False):
        lib.glide_gemm_bf16.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        lib.glide_gemm_bf16.restype = C.c_int
        lib.glide_im2col3_bf16.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 5 + [C.c_void_p]
        lib.glide_im2col3_bf16.restype = C.c_int
        lib.glide_col2im3_f32.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 5 + [C.c_void_p]
        lib.glide_col2im3_f32.restype = C.c_int
        lib.glide_transpose_bf16.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        lib.glide_transpose_bf16.restype = C.c_int
        lib.glide_conv3x3_bf16.argtypes = [C.c_void_p] + [C.c_int] * 4 + [C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                                                          C.c_int, C.c_void_p, C.c_int, C.c_int,
                                                                          C.c_void_p, C.c_void_p]
        lib.glide_conv3x3_bf16.restype = C.c_int
        lib._guess_sigs = True
    return lib


_ERR = {}


def _err_flag(device):
    t = _ERR.get(device)
    if t is None:
        t = torch.zeros(1, dtype=torch.int32, device=device)
        _ERR[device] = t
    return t


def gemm(A, B, out, bias=None, relu=False, out_mode=0):
    """out (+)= A @ B.T on the tensor cores (A: M x K, B: N x K, both BF16)."""
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16
    assert A.is_contiguous() and B.is_contiguous() and out.is_contiguous()
    M, K = A.shape
    Nn = B.shape[0]
    rc = _lib().glide_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, out.data_ptr(), Nn, M, Nn, K,
                                None if bias is None else bias.data_ptr(), int(relu), int(out_mode),
                                _err_flag(A.device).data_ptr(), N.stream_handle())
    N.check(rc, "tensor-core gemm")
    return out


def conv3x3(x, Wb, out, bias=None, relu=False, out_mode=1):
    """out (+)= conv3x3(x) on the tensor cores as an implicit GEMM (no im2col
    buffer): x NHWC BF16 with C % 8 == 0, Wb (Cout, 9C) BF16."""
    assert x.dtype == torch.bfloat16 and Wb.dtype == torch.bfloat16
    assert x.is_contiguous() and Wb.is_contiguous() and out.is_contiguous()
    Bn, H, W, Cc = x.shape
    Nn = Wb.shape[0]
    rc = _lib().glide_conv3x3_bf16(x.data_ptr(), Bn, H, W, Cc, Wb.data_ptr(), Wb.shape[1], out.data_ptr(), Nn, Nn,
                                   None if bias is None else bias.data_ptr(), int(relu), int(out_mode),
                                   _err_flag(x.device).data_ptr(), N.stream_handle())
    N.check(rc, "tensor-core conv3x3")
    return out


def im2col3(x):
    Bn, H, W, Cc = x.shape
    col = torch.empty((Bn * H * W, 9 * Cc), dtype=torch.bfloat16, device=x.device)
    N.check(_lib().glide_im2col3_bf16(x.data_ptr(), col.data_ptr(), Bn, H, W, Cc, 9 * Cc, N.stream_handle()),
            "im2col")
    return col


def col2im3(dcol, shape):
    Bn, H, W, Cc = shape
    dx = torch.empty((Bn, H, W, Cc), dtype=torch.float32, device=dcol.device)
    N.check(_lib().glide_col2im3_f32(dcol.data_ptr(), dx.data_ptr(), Bn, H, W, Cc, 9 * Cc, N.stream_handle()),
            "col2im")
    return dx


def transpose(x):
    R, Cc = x.shape
    y = torch.empty((Cc, R), dtype=torch.bfloat16, device=x.device)
    N.check(_lib().glide_transpose_bf16(x.data_ptr(), y.data_ptr(), R, Cc, N.stream_handle()), "transpose")
    return y


def conv3x3_relu(x, W, b, relu=True):
    """relu(conv3x3(x, W) + b).  With autograd recording (training) this is
    Conv3x3ReLU, which keeps the im2col matrix for the weight gradient; without
    (inference) the im2col is gathered inside the GEMM when Cin % 8 == 0, with a
    bit-identical result."""
    Bn, H, Wd, Cin = x.shape
    if (torch.is_grad_enabled() and (x.requires_grad or W.requires_grad or b.requires_grad)) or Cin % 8 != 0:
        return Conv3x3ReLU.apply(x, W, b, relu)
    Cout = W.shape[0]
    y = torch.empty((Bn * H * Wd, Cout), dtype=torch.bfloat16, device=x.device)
    conv3x3(x.contiguous(), W.detach().to(torch.bfloat16).contiguous(), y, bias=b.detach(), relu=relu, out_mode=1)
    return y.view(Bn, H, Wd, Cout)


class Conv3x3ReLU(torch.autograd.Function):
    """y = relu(conv3x3(x, W) + b); x NHWC BF16, W (Cout, 9*Cin) FP32 master."""

    @staticmethod
    def forward(ctx, x, W, b, relu: bool):
        Bn, H, Wd, Cin = x.shape
        Cout = W.shape[0]
        x = x.contiguous()
        Wb = W.to(torch.bfloat16).contiguous()
        y = torch.empty((Bn * H * Wd, Cout), dtype=torch.bfloat16, device=x.device)
        col = im2col3(x)
        gemm(col, Wb, y, bias=b, relu=relu, out_mode=1)
        ctx.save_for_backward(col, Wb, y)
        ctx.shape = (Bn, H, Wd, Cin)
        ctx.relu = relu
        return y.view(Bn, H, Wd, Cout)

    @staticmethod
    def backward(ctx, gy):
        col, Wb, y = ctx.saved_tensors
        Bn, H, Wd, Cin = ctx.shape
        Cout = Wb.shape[0]
        P = Bn * H * Wd
        g = gy.reshape(P, Cout).float()
        if ctx.relu:
            g = g * (y > 0)
        gz = g.to(torch.bfloat16).contiguous()
        # weight gradient: dW (Cout x 9Cin) = gz^T (Cout x P) . col (P x 9Cin)
        dW = torch.zeros((Cout, 9 * Cin), dtype=torch.float32, device=gy.device)
        gemm(transpose(gz), transpose(col), dW, out_mode=0)
        db = g.sum(0)
        # data gradient: dcol (P x 9Cin) = gz (P x Cout) . W (Cout x 9Cin)
        dcol = torch.empty((P, 9 * Cin), dtype=torch.float32, device=gy.device)
        gemm(gz, transpose(Wb), dcol, out_mode=0)
        dx = col2im3(dcol, (Bn, H, Wd, Cin))
        return dx.to(torch.bfloat16), dW, db, None


class Conv1x1(torch.autograd.Function):
    """Linear head y = x . W^T + b per pixel (x NHWC BF16, y FP32)."""

    @staticmethod
    def forward(ctx, x, W, b):
        Bn, H, Wd, Cin = x.shape
        Cout = W.shape[0]
        xf = x.reshape(-1, Cin).contiguous()
        Wb = W.to(torch.bfloat16).contiguous()
        y = torch.empty((xf.shape[0], Cout), dtype=torch.float32, device=x.device)
        gemm(xf, Wb, y, bias=b, out_mode=0)
        ctx.save_for_backward(xf, Wb)
        ctx.shape = (Bn, H, Wd, Cin)
        return y.view(Bn, H, Wd, Cout)

    @staticmethod
    def backward(ctx, gy):
        xf, Wb = ctx.saved_tensors
        Bn, H, Wd, Cin = ctx.shape
        Cout = Wb.shape[0]
        g = gy.reshape(-1, Cout).float()
        gz = g.to(torch.bfloat16).contiguous()
        dW = torch.zeros((Cout, Cin), dtype=torch.float32, device=gy.device)
        gemm(transpose(gz), transpose(xf), dW, out_mode=0)
        dx = torch.empty((xf.shape[0], Cin), dtype=torch.float32, device=gy.device)
        gemm(gz, transpose(Wb), dx, out_mode=0)
        return dx.view(Bn, H, Wd, Cin).to(torch.bfloat16), dW, g.sum(0)


def _pool(x):
    Bn, H, W, Cc = x.shape
    return x.view(Bn, H // 2, 2, W // 2, 2, Cc).float().mean((2, 4)).to(torch.bfloat16)


def _up(x):
    return x.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)


class UNet(torch.nn.Module):
    """4-level, 32-base-channel U-Net (NHWC, BF16 activations)."""

    def __init__(self, base=32, levels=4, in_ch=IN_CH, out_ch=2, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        chans = [base * 2 ** k for k in range(levels)]
        self.levels = levels
        self.ws = torch.nn.ParameterList()
        self.bs = torch.nn.ParameterList()
        self.plan = []   # (cin, cout) of each 3x3 conv, in order

        def add(cin, cout):
            w = torch.randn(cout, 9 * cin, generator=g) * math.sqrt(2.0 / (9 * cin))
            self.ws.append(torch.nn.Parameter(w))
            self.bs.append(torch.nn.Parameter(torch.zeros(cout)))
            self.plan.append((cin, cout))

        cin = in_ch
        for k in range(levels):            # encoder
            add(cin, chans[k])
            add(chans[k], chans[k])
            cin = chans[k]
        for k in range(levels - 2, -1, -1):  # decoder
            add(cin + chans[k], chans[k])
            add(chans[k], chans[k])
            cin = chans[k]
        self.head_w = torch.nn.Parameter(torch.randn(out_ch, cin, generator=g) * math.sqrt(1.0 / cin))
        self.head_b = torch.nn.Parameter(torch.zeros(out_ch))

    def forward(self, x):
        """x: (B, H, W, IN_CH) BF16, H and W divisible by 2**(levels-1)."""
        i = 0
        skips = []
        for k in range(self.levels):
            x = conv3x3_relu(x, self.ws[i], self.bs[i]); i += 1
            x = conv3x3_relu(x, self.ws[i], self.bs[i]); i += 1
            if k < self.levels - 1:
                skips.append(x)
                x = _pool(x)
        for k in range(self.levels - 2, -1, -1):
            x = torch.cat([_up(x), skips[k]], dim=3)
            x = conv3x3_relu(x, self.ws[i], self.bs[i]); i += 1
            x = conv3x3_relu(x, self.ws[i], self.bs[i]); i += 1
        return Conv1x1.apply(x, self.head_w, self.head_b)

    def flops(self, H, W):
        """Multiply-add FLOPs of one forward pass on an H x W input (x2 per MAC)."""
        tot = 0.0
        k = 0
        hh, ww = H, W
        for lv in range(self.levels):
            for _ in range(2):
                cin, cout = self.plan[k]
                tot += 2.0 * 9 * cin * cout * hh * ww
                k += 1
            if lv < self.levels - 1:
                hh, ww = hh // 2, ww // 2
        for lv in range(self.levels - 2, -1, -1):
            hh, ww = hh * 2, ww * 2
            for _ in range(2):
                cin, cout = self.plan[k]
                tot += 2.0 * 9 * cin * cout * hh * ww
                k += 1
        return tot + 2.0 * self.head_w.numel() * H * W


# ---------------------------------------------------------------------------
# features, targets and the guess interface
# ---------------------------------------------------------------------------

def features(H, bed, beta, B):
    """(…, ny, nx) fields -> (B, ny, nx, IN_CH) BF16 normalised inputs."""
    def b3(t):
        t = torch.as_tensor(t)
        return t.unsqueeze(0) if t.dim() == 2 else t
    H, bed, beta, B = (b3(t).float() for t in (H, bed, beta, B))
    logb = torch.log(torch.clamp(beta, min=1e-8))
    x = torch.stack([H / 1000.0, bed / 1000.0, (logb + 2.2) / 0.7, B / 35.0], dim=-1)
    pad = torch.zeros(x.shape[:-1] + (IN_CH - x.shape[-1],), device=x.device)
    return torch.cat([x, pad], dim=-1).to(torch.bfloat16).contiguous()


def cell_velocities(u, v):
    """Face velocities -> cell-centred (…, ny, nx, 2) / VEL_SCALE."""
    uc = 0.5 * (u[..., :, 1:] + u[..., :, :-1])
    vc = 0.5 * (v[..., 1:, :] + v[..., :-1, :])
    return torch.stack([uc, vc], dim=-1) / VEL_SCALE


def faces_from_cells(pred):
    """(…, ny, nx, 2) cell velocities (scaled) -> staggered (u, v) in m/a."""
    uc = pred[..., 0] * VEL_SCALE
    vc = pred[..., 1] * VEL_SCALE
    u = torch.cat([uc[..., :, :1], 0.5 * (uc[..., :, 1:] + uc[..., :, :-1]), uc[..., :, -1:]], dim=-1)
    v = torch.cat([vc[..., :1, :], 0.5 * (vc[..., 1:, :] + vc[..., :-1, :]), vc[..., -1:, :]], dim=-2)
    return u, v


class GuessModel:
    """Trained network + the IcePhysics guess interface."""

    def __init__(self, net: UNet):
        self.net = net

    @torch.no_grad()
    def predict(self, H, bed, beta, B):
        x = features(H, bed, beta, B)
        pred = self.net(x)
        u, v = faces_from_cells(pred.float())
        if u.shape[0] == 1:
            u, v = u[0], v[0]
        return u.double(), v.double()

    def save(self, path=DEFAULT_WEIGHTS):
        torch.save(self.net.state_dict(), path)


def load_default_model(path=DEFAULT_WEIGHTS, device="cuda"):
    """The trained guess shipped with the package, or None when absent."""
    if not Path(path).exists():
        return None
    net = UNet()
    net.load_state_dict(torch.load(path, map_location="cpu"))
    return GuessModel(net.to(device))
