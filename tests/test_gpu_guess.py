"""Learned-guess network: tensor-core convolution gradients vs a CPU oracle,
and the fallback rule of the guess.

The CPU oracle is torch's FP32 conv2d / autograd on the same BF16-rounded
inputs and weights.  Tolerance: relative max error <= 2e-2 for outputs and
gradients (BF16 operands, BF16 activations between the products, FP32
accumulation).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return (a.float().cpu() - b.float().cpu()).abs().max().item() / (b.float().abs().max().item() + 1e-12)


def test_conv3x3_forward_backward_vs_cpu():
    from glide_b200.guess import Conv3x3ReLU
    torch.manual_seed(0)
    Bn, H, W, Cin, Cout = 2, 16, 24, 16, 32
    x = torch.randn(Bn, H, W, Cin, device="cuda").bfloat16().requires_grad_(True)
    Wm = (torch.randn(Cout, 9 * Cin, device="cuda") * 0.1).requires_grad_(True)
    b = (torch.randn(Cout, device="cuda") * 0.1).requires_grad_(True)
    y = Conv3x3ReLU.apply(x, Wm, b, True)
    gy = torch.randn_like(y, dtype=torch.float32)
    y.float().backward(gy)
    # CPU oracle on the same BF16 values
    xc = x.detach().float().cpu().permute(0, 3, 1, 2).requires_grad_(True)
    wc = Wm.detach().bfloat16().float().cpu().reshape(Cout, 3, 3, Cin).permute(0, 3, 1, 2).contiguous().requires_grad_(True)
    bc = b.detach().cpu().requires_grad_(True)
    yc = torch.relu(torch.nn.functional.conv2d(xc, wc, bc, padding=1))
    yc.backward(gy.cpu().permute(0, 3, 1, 2))
    assert _rel(y.permute(0, 3, 1, 2), yc) <= 2e-2
    assert _rel(x.grad.permute(0, 3, 1, 2), xc.grad) <= 2e-2
    dW_ref = wc.grad.permute(0, 2, 3, 1).reshape(Cout, 9 * Cin)
    assert _rel(Wm.grad, dW_ref) <= 2e-2
    assert _rel(b.grad, bc.grad) <= 2e-2


def test_unet_inference_matches_training_forward_bitwise():
    """Without autograd the convolutions gather the im2col inside the GEMM;
    the output is bit-identical to the recorded (im2col-matrix) forward."""
    from glide_b200.guess import UNet, features
    torch.manual_seed(1)
    net = UNet().cuda()
    H = torch.rand(1, 128, 96, device="cuda") * 1000
    x = features(H, H * 0.1, torch.full_like(H, 0.1), torch.full_like(H, 35.0))
    y_train = net(x)
    assert y_train.requires_grad
    with torch.no_grad():
        y_inf = net(x)
    assert torch.equal(y_train.detach(), y_inf)


def test_unet_forward_shapes_and_gradients_flow():
    from glide_b200.guess import UNet, features
    net = UNet().cuda()
    H = torch.rand(2, 64, 64, device="cuda") * 1000
    x = features(H, H * 0, torch.full_like(H, 0.1), torch.full_like(H, 35.0))
    y = net(x)
    assert y.shape == (2, 64, 64, 2)
    loss = (y ** 2).mean()
    loss.backward()
    assert all(p.grad is not None and torch.isfinite(p.grad).all() for p in net.parameters())


def test_bad_guess_falls_back_to_plain_solve():
    """A corrupted (NaN-poisoned) guess is rejected by the first-cycle rule
    and the step still reaches the tolerance from the plain start."""
    from glide_b200 import IcePhysics, SolverSettings
    from glide_b200.synthetic import dome_sheet_case
    c = dome_sheet_case(3, n=128, dx=8000.0, n_levels=4)
    ph = IcePhysics(128, 128, c.dx, n_levels=4, precision="fp64", settings=SolverSettings(shift=0.0, err_threshold=1e-7))
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    bu = torch.zeros((128, 129), dtype=torch.float64)
    bu[40:60, 40:60] = float("nan")
    bad = (bu, torch.zeros((129, 128), dtype=torch.float64))
    ph.forward(c.dt, tol=1e-6, max_vcycles=30, guess=bad)
    assert ph.last_info["fallback"] is True
    assert ph.last_info["rel_residual"] <= 1e-6


def test_learned_guess_gain_on_held_out_patches():
    """What the trained model gains: on held-out 256x256 patches of its training
    family (seeds far from the training range), its velocity is within 15 % of
    the converged FP64 solution (norm-wise; measured 4.5-9.4 %), where the zero
    start is 100 % off.  The time-to-tolerance effect is measured by bench.py."""
    from glide_b200 import IcePhysics, SolverSettings
    from glide_b200.guess import load_default_model
    from glide_b200.synthetic import training_patch_case
    model = load_default_model()
    for seed in (50_007, 50_008, 50_009):
        c = training_patch_case(seed)
        ph = IcePhysics(c.ny, c.nx, c.dx, n_levels=4, thklim=c.thklim, precision="fp64",
                        settings=SolverSettings(shift=0.0, err_threshold=1e-7))
        ph.set_geometry(c.bed, c.thickness)
        ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
        dev = {k: torch.as_tensor(v, device="cuda") for k, v in
               (("H", c.thickness), ("bed", c.bed), ("beta", c.beta), ("B", c.B))}
        gu, gv = model.predict(dev["H"], dev["bed"], dev["beta"], dev["B"])
        ph.forward(c.dt, tol=1e-9, max_vcycles=60, update_geometry=False)
        assert ph.last_info["rel_residual"] <= 1e-9
        us, vs = ph.grid.u, ph.grid.v
        err = torch.sqrt(((gu - us) ** 2).sum() + ((gv - vs) ** 2).sum()) / torch.sqrt((us ** 2).sum() + (vs ** 2).sum())
        assert err.item() <= 0.15, (seed, err.item())
