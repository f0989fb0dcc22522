"""Operator parity: sm_100a kernels vs the FP64 NumPy oracle.

Tolerances (norm-wise relative error ||a-b|| / ||b||):
  FP64 kernels  <= 1e-10   (same formulas, different summation order)
  FP32 kernels  <= 2e-5    (single application of one operator)
Sizes cover tile edges: 32 (multiple of the 32x16 tile), 40x24 (ragged),
and a batch of 3 problems.
"""
import numpy as np
import pytest
import torch

from conftest import random_state

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 2e-5}


def _rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _grid(st, precision, gl_derivatives=False, nb=1):
    import torch
    from glide_b200.grid import Grid
    dt = torch.float64 if precision == "fp64" else torch.float32
    ny, nx = st["H"].shape[-2:]
    g = Grid(ny, nx, st["dx"], dt=st["dt"], dtype=dt, gl_derivatives=gl_derivatives, nb=nb)
    for k in ("u", "v", "H", "bed", "B", "beta", "mask", "gamma", "f_u", "f_v", "f_H", "d_u", "d_v", "d_H"):
        getattr(g, k).copy_(torch.as_tensor(st[k]))
    return g


def _np(t):
    return t.detach().double().cpu().numpy()


def _state(shape=(32, 32), seed=0):
    ny, nx = shape
    n = max(ny, nx)
    st = random_state(n=n, seed=seed)
    if (ny, nx) != (n, n):
        for k in list(st):
            if isinstance(st[k], np.ndarray):
                a = st[k]
                rows = ny + (a.shape[0] - n)
                cols = nx + (a.shape[1] - n)
                st[k] = np.ascontiguousarray(a[:rows, :cols])
    return st


def _params(gl=False):
    from oracle.ssa import Params
    return Params(gl_derivatives=gl)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(32, 32), (24, 40), (33, 47), (70, 100), (5, 3), (130, 61)])
def test_residual(precision, shape):
    from oracle import ssa
    st = _state(shape)
    g = _grid(st, precision)
    g.compute_residual()
    ref = ssa.residual(st["u"], st["v"], st["H"], st["f_u"], st["f_v"], st["f_H"], st["bed"], st["B"], st["beta"],
                       st["mask"], st["gamma"], _params(), st["dx"], st["dt"])
    for a, b in zip((g.r_u, g.r_v, g.r_H), ref):
        assert _rel(_np(a), b) <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("gl", [False, True])
@pytest.mark.parametrize("shape", [(24, 40), (32, 32), (33, 47), (70, 100), (5, 3), (130, 61)])
def test_jvp(precision, gl, shape):
    from oracle import ssa
    st = _state(shape, seed=1)
    g = _grid(st, precision, gl_derivatives=gl)
    g.compute_jvp()
    ref = ssa.jvp(st["u"], st["v"], st["H"], st["d_u"], st["d_v"], st["d_H"], st["bed"], st["B"], st["beta"],
                  st["mask"], st["gamma"], _params(gl), st["dx"], st["dt"])
    for a, b in zip((g.j_u, g.j_v, g.j_H), ref):
        assert _rel(_np(a), b) <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(24, 40), (70, 100), (5, 3)])
def test_jvp_add(precision, shape):
    """glide_jvp_add writes base + J d: against the oracle's J d plus base, and
    within rounding of the base plus the plain JVP's output."""
    from oracle import ssa
    st = _state(shape, seed=5)
    g = _grid(st, precision, gl_derivatives=True)
    base = torch.randn(g.U.shape, dtype=torch.float64, generator=torch.Generator().manual_seed(3)) * 1e-2
    base = base.to(g.U.device, g.dtype)
    out = torch.full_like(g.U, float("nan"))
    g.jvp_add(base, out)
    g.compute_jvp()
    ref = ssa.jvp(st["u"], st["v"], st["H"], st["d_u"], st["d_v"], st["d_H"], st["bed"], st["B"], st["beta"],
                  st["mask"], st["gamma"], _params(True), st["dx"], st["dt"])
    ou, ov, oH = g._vec_to_fields(out)
    bu, bv, bH = g._vec_to_fields(base)
    for o, b_, j, r in zip((ou, ov, oH), (bu, bv, bH), (g.j_u, g.j_v, g.j_H), ref):
        assert _rel(_np(o), _np(b_) + r) <= TOL[precision]
        eps = torch.finfo(g.dtype).eps
        assert float((o - (b_ + j)).abs().max()) <= 8 * eps * float((b_.abs() + j.abs()).max())


def test_jvp_add_rejects_aliasing():
    import ctypes as C
    from glide_b200 import _native as N
    st = _state((24, 40), seed=5)
    g = _grid(st, "fp32")
    a = g.level_args()
    p = [t.data_ptr() for t in (g.d_u, g.d_v, g.d_H, g.r_u, g.r_v, g.r_H)]
    assert N.load().glide_jvp_add(C.byref(a), *p, p[3], p[4], p[5], N.stream_handle()) == -2


def test_jvp_batch_matches_single():
    """A batch of 3 problems gives the same JVP as 3 single calls."""
    from glide_b200.grid import Grid
    sts = [_state((33, 47), seed=s) for s in (20, 21, 22)]
    g = Grid(33, 47, sts[0]["dx"], dt=10.0, dtype=torch.float32, nb=3, gl_derivatives=True)
    for k in ("u", "v", "H", "bed", "B", "beta", "mask", "gamma", "d_u", "d_v", "d_H"):
        getattr(g, k).copy_(torch.as_tensor(np.stack([s[k] for s in sts])))
    g.compute_jvp()
    for b, st in enumerate(sts):
        g1 = _grid(st, "fp32", gl_derivatives=True)
        g1.compute_jvp()
        assert torch.equal(g.j_u[b], g1.j_u) and torch.equal(g.j_v[b], g1.j_v) and torch.equal(g.j_H[b], g1.j_H)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("gl,exact", [(False, False), (True, False), (True, True)])
@pytest.mark.parametrize("shape", [(32, 32), (24, 40), (33, 47), (70, 100), (5, 3), (130, 61)])
def test_vjp(precision, gl, exact, shape):
    import torch
    from oracle import ssa
    st = _state(shape, seed=2)
    g = _grid(st, precision, gl_derivatives=gl)
    g.lambda_u.copy_(torch.as_tensor(st["d_u"]))
    g.lambda_v.copy_(torch.as_tensor(st["d_v"]))
    g.lambda_H.copy_(torch.as_tensor(st["d_H"]))
    g.compute_vjp(exact_boundary=exact)
    ref = ssa.vjp(st["u"], st["v"], st["H"], st["d_u"], st["d_v"], st["d_H"], st["bed"], st["B"], st["beta"],
                  st["mask"], st["gamma"], _params(gl), st["dx"], st["dt"], exact_boundary=exact)
    for a, b in zip((g.l_u, g.l_v, g.l_H), ref):
        assert _rel(_np(a), b) <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vjp_residual_form(precision):
    """glide_vjp with f writes f - lambda^T J (the adjoint residual)."""
    import ctypes as C
    from glide_b200 import _native as N
    st = _state((70, 100), seed=6)
    g = _grid(st, precision, gl_derivatives=True)
    g.lambda_u.copy_(torch.as_tensor(st["d_u"]))
    g.lambda_v.copy_(torch.as_tensor(st["d_v"]))
    g.lambda_H.copy_(torch.as_tensor(st["d_H"]))
    g.compute_vjp(exact_boundary=True)
    a = g.level_args()
    out = [torch.full_like(t, float("nan")) for t in (g.l_u, g.l_v, g.l_H)]
    N.check(N.load().glide_vjp(C.byref(a), g.lambda_u.data_ptr(), g.lambda_v.data_ptr(), g.lambda_H.data_ptr(),
                               g.f_u.data_ptr(), g.f_v.data_ptr(), g.f_H.data_ptr(), out[0].data_ptr(),
                               out[1].data_ptr(), out[2].data_ptr(), 1, N.stream_handle()), "vjp")
    eps = torch.finfo(g.dtype).eps
    for o, f, l in zip(out, (g.f_u, g.f_v, g.f_H), (g.l_u, g.l_v, g.l_H)):
        assert float((o - (f - l)).abs().max()) <= 8 * eps * float((f.abs() + l.abs()).max())


def test_vjp_batch_matches_single():
    """A batch of 3 problems gives the same VJP as 3 single calls."""
    from glide_b200.grid import Grid
    sts = [_state((33, 47), seed=s) for s in (30, 31, 32)]
    g = Grid(33, 47, sts[0]["dx"], dt=10.0, dtype=torch.float32, nb=3, gl_derivatives=True)
    for k in ("u", "v", "H", "bed", "B", "beta", "mask", "gamma"):
        getattr(g, k).copy_(torch.as_tensor(np.stack([s[k] for s in sts])))
    g.lambda_u.copy_(torch.as_tensor(np.stack([s["d_u"] for s in sts])))
    g.lambda_v.copy_(torch.as_tensor(np.stack([s["d_v"] for s in sts])))
    g.lambda_H.copy_(torch.as_tensor(np.stack([s["d_H"] for s in sts])))
    g.compute_vjp(exact_boundary=True)
    for b, st in enumerate(sts):
        g1 = _grid(st, "fp32", gl_derivatives=True)
        g1.lambda_u.copy_(torch.as_tensor(st["d_u"]))
        g1.lambda_v.copy_(torch.as_tensor(st["d_v"]))
        g1.lambda_H.copy_(torch.as_tensor(st["d_H"]))
        g1.compute_vjp(exact_boundary=True)
        assert torch.equal(g.l_u[b], g1.l_u) and torch.equal(g.l_v[b], g1.l_v) and torch.equal(g.l_H[b], g1.l_H)


def test_vjp_dot_jvp_fp64():
    """<lambda, J d> == <J^T lambda, d> with the exact-boundary VJP."""
    import torch
    st = _state((24, 40), seed=3)
    g = _grid(st, "fp64", gl_derivatives=True)
    g.compute_jvp()
    g.lambda_u.copy_(torch.as_tensor(st["f_u"]))
    g.lambda_v.copy_(torch.as_tensor(st["f_v"]))
    g.lambda_H.copy_(torch.as_tensor(st["f_H"]))
    g.compute_vjp(exact_boundary=True)
    a = float((g.lambda_u * g.j_u).sum() + (g.lambda_v * g.j_v).sum() + (g.lambda_H * g.j_H).sum())
    b = float((g.l_u * g.d_u).sum() + (g.l_v * g.d_v).sum() + (g.l_H * g.d_H).sum())
    assert abs(a - b) <= 1e-12 * abs(a)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("exact", [False, True])
def test_grad_beta(precision, exact):
    import torch
    from oracle import ssa
    st = _state((24, 40), seed=4)
    g = _grid(st, precision)
    g.lambda_u.copy_(torch.as_tensor(st["d_u"]))
    g.lambda_v.copy_(torch.as_tensor(st["d_v"]))
    grad = g.compute_grad_beta(exact_boundary=exact)
    ref = ssa.grad_beta(st["u"], st["v"], st["H"], st["d_u"], st["d_v"], st["bed"], st["beta"], _params(),
                        exact_boundary=exact)
    assert _rel(_np(grad), ref) <= TOL[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shift,step,n_newton,pivot", [(1.0, 0.25, 10, False), (0.0, 0.25, 10, False),
                                                      (0.0, 1.0, 2, False), (0.0, 0.25, 10, True)])
def test_vanka_sweep(precision, shift, step, n_newton, pivot):
    """One sweep vs the oracle; step 0.25 is the reference smoother, step 1.0
    with 2 iterations the finishing sweeps of the tolerance solver, pivot the
    row-pivoted local solve."""
    from oracle.vanka import vanka_deltas
    st = _state((32, 32), seed=5)
    st["u"] *= 0.02
    st["v"] *= 0.02
    g = _grid(st, precision)
    g.vanka_sweep(1, n_inner=n_newton, omega=0.5, shift=shift, step=step, pivot=pivot)
    du, dv, dH = vanka_deltas(st["u"], st["v"], st["H"], st["f_u"], st["f_v"], st["f_H"], st["bed"], st["B"],
                              st["beta"], st["gamma"], _params(), st["dx"], st["dt"], n_newton, shift=shift, step=step,
                              pivot=pivot)
    tol = TOL[precision] * (1 if precision == "fp64" else 20)
    for a, x0, d in zip((g.u, g.v, g.H), (st["u"], st["v"], st["H"]), (du, dv, dH)):
        assert _rel(_np(a) - x0, 0.5 * d) <= tol


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vanka_ex_reference_step_is_the_reference_entry_point(precision):
    """glide_vanka_sweeps_ex with step 0.25 is bit-identical to glide_vanka_sweeps."""
    import ctypes as C
    st = _state((40, 24), seed=6)
    st["u"] *= 0.02
    st["v"] *= 0.02
    a, b = _grid(st, precision), _grid(st, precision)
    a.vanka_sweep(2, n_inner=10, omega=0.5, shift=1.0)
    args = b.level_args()
    rc = b._lib.glide_vanka_sweeps(C.byref(args), b.f_u.data_ptr(), b.f_v.data_ptr(), b.f_H.data_ptr(), 2, 10, 0.5,
                                   1.0, None, None, b._scratch.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    assert torch.equal(a.U, b.U)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vanka_local_gating(precision):
    import torch
    from oracle.vanka import local_cell_on, vanka_deltas
    st = _state((40, 40), seed=6)
    st["u"] *= 0.02
    st["v"] *= 0.02
    g = _grid(st, precision)
    em = np.zeros((40, 40))
    em[3, 20] = 1.0      # inside block (0,1)'s window
    em[27, 13] = 1.0     # on a block ring: activates two blocks
    g.error_mask.copy_(torch.as_tensor(em))
    g.vanka_sweep_local(1, n_inner=10, omega=0.5)
    on = local_cell_on(em)
    du, dv, dH = vanka_deltas(st["u"], st["v"], st["H"], st["f_u"], st["f_v"], st["f_H"], st["bed"], st["B"],
                              st["beta"], st["gamma"], _params(), st["dx"], st["dt"], 10, cell_on=on)
    tol = TOL[precision] * (1 if precision == "fp64" else 20)
    for a, x0, d in zip((g.u, g.v, g.H), (st["u"], st["v"], st["H"]), (du, dv, dH)):
        assert _rel(_np(a) - x0, 0.5 * d) <= tol
    assert on.sum() < on.size  # gating actually skipped cells


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vanka_adjoint(precision):
    import torch
    from oracle import ssa
    from oracle.vanka import vanka_adjoint_color
    st = _state((32, 32), seed=7)
    g = _grid(st, precision)
    g.lambda_u.copy_(torch.as_tensor(st["d_u"]))
    g.lambda_v.copy_(torch.as_tensor(st["d_v"]))
    g.lambda_H.copy_(torch.as_tensor(st["d_H"]))
    g.f_adj_u.copy_(torch.as_tensor(st["f_u"]))
    g.f_adj_v.copy_(torch.as_tensor(st["f_v"]))
    g.f_adj_H.copy_(torch.as_tensor(st["f_H"]))
    p = _params()
    lu, lv, lH = st["d_u"], st["d_v"], st["d_H"]
    for color in (0, 1):
        g.compute_adjoint_residual()
        g.vanka_smooth_adjoint(color, omega=1.0)
        vu, vv, vH = ssa.vjp(st["u"], st["v"], st["H"], lu, lv, lH, st["bed"], st["B"], st["beta"], st["mask"],
                             st["gamma"], p, st["dx"], st["dt"])
        r = (st["f_u"] - vu, st["f_v"] - vv, st["f_H"] - vH)
        lu, lv, lH = vanka_adjoint_color(lu, lv, lH, st["mask"], r, st["u"], st["v"], st["H"], st["bed"], st["B"],
                                         st["beta"], st["gamma"], p, st["dx"], st["dt"], color, 1.0)
    tol = TOL[precision] * (1 if precision == "fp64" else 50)
    for a, b in zip((g.lambda_u, g.lambda_v, g.lambda_H), (lu, lv, lH)):
        assert _rel(_np(a), b) <= tol


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_transfers(precision):
    import torch
    from glide_b200 import kernels as K
    from oracle import multigrid as O
    rng = np.random.default_rng(8)
    dt = torch.float64 if precision == "fp64" else torch.float32
    uf, vf, hf = rng.standard_normal((16, 25)), rng.standard_normal((17, 24)), rng.standard_normal((16, 24))
    uc, vc, hc = rng.standard_normal((8, 13)), rng.standard_normal((9, 12)), rng.standard_normal((8, 12))
    T = lambda a: torch.as_tensor(a, dtype=dt, device="cuda")
    tol = TOL[precision]
    assert _rel(_np(K.restrict_vfacet(T(uf))), O.restrict_u(uf)) <= tol
    assert _rel(_np(K.restrict_hfacet(T(vf))), O.restrict_v(vf)) <= tol
    assert _rel(_np(K.restrict_cell_centered(T(hf))), O.restrict_cell(hf)) <= tol
    assert _rel(_np(K.restrict_max_pool(T(hf))), O.restrict_max_pool(hf)) <= tol
    assert _rel(_np(K.prolongate_vfacet(T(uc), smooth=True)), O.prolong_u_bilinear(uc)) <= tol
    assert _rel(_np(K.prolongate_vfacet(T(uc), smooth=False)), O.prolong_u_linear(uc)) <= tol
    assert _rel(_np(K.prolongate_hfacet(T(vc), smooth=True)), O.prolong_v_bilinear(vc)) <= tol
    assert _rel(_np(K.prolongate_hfacet(T(vc), smooth=False)), O.prolong_v_linear(vc)) <= tol
    assert _rel(_np(K.prolongate_cell_centered(T(hc), smooth=True)), O.prolong_cell_bilinear(hc)) <= tol
    assert _rel(_np(K.prolongate_cell_centered(T(hc), smooth=False)), O.prolong_cell_inject(hc)) <= tol


def test_batch_matches_single():
    """A batch of 3 problems gives the same residual as 3 single calls."""
    import torch
    from glide_b200.grid import Grid
    sts = [_state((24, 40), seed=s) for s in (10, 11, 12)]
    g = Grid(24, 40, sts[0]["dx"], dt=10.0, dtype=torch.float64, nb=3)
    for k in ("u", "v", "H", "bed", "B", "beta", "mask", "gamma", "f_u", "f_v", "f_H"):
        getattr(g, k).copy_(torch.as_tensor(np.stack([s[k] for s in sts])))
    g.compute_residual()
    for b, st in enumerate(sts):
        g1 = _grid(st, "fp64")
        g1.compute_residual()
        assert torch.equal(g.r_u[b], g1.r_u) and torch.equal(g.r_v[b], g1.r_v) and torch.equal(g.r_H[b], g1.r_H)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vanka_failed_local_solve_leaves_cell_unchanged(precision):
    """A non-finite right-hand side at one face makes the two cells sharing it
    fail their local solve: those cells keep their values, every other update
    matches the sweep without the bad value, and nothing turns non-finite."""
    st = _state((24, 40), seed=7)
    st["u"] *= 0.02
    st["v"] *= 0.02
    good, bad = _grid(st, precision), _grid(st, precision)
    i, j = 10, 17
    bad.f_u[i, j] = float("nan")
    for g in (good, bad):
        g.vanka_sweep(1, n_inner=2, omega=0.5, shift=0.0, step=1.0)
    assert torch.isfinite(bad.U).all()
    assert bad.H[i, j - 1] == torch.as_tensor(st["H"][i, j - 1], dtype=bad.dtype)
    assert bad.H[i, j] == torch.as_tensor(st["H"][i, j], dtype=bad.dtype)
    far = torch.ones_like(bad.H, dtype=torch.bool)
    far[max(i - 2, 0):i + 3, max(j - 3, 0):j + 3] = False
    assert torch.equal(bad.H[far], good.H[far])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vanka_linear_sweep_vs_oracle(precision):
    """Linear Vanka (defect-correction sweeps): factors at U, one additive
    update of d for the linear residual rho, against the oracle's restatement
    (norm-wise relative 1e-10 in FP64, 2e-4 in FP32)."""
    from oracle.vanka import vanka_linear_update
    st = _state((24, 40), seed=8)
    st["u"] *= 0.02
    st["v"] *= 0.02
    g = _grid(st, precision)
    rng = np.random.default_rng(9)
    rho = rng.standard_normal(g.U.numel())
    d = rng.standard_normal(g.U.numel()) * 0.1
    g.vanka_lu(shift=0.0)
    rho_t = torch.as_tensor(rho, dtype=g.dtype, device="cuda")
    d_t = torch.as_tensor(d, dtype=g.dtype, device="cuda")
    d0 = d_t.clone()
    g.vanka_linear_sweep(rho_t, d_t, omega=0.5)
    ru, rv, rH = (x.detach().cpu().numpy().astype(float) for x in g._vec_to_fields(torch.as_tensor(rho, device="cuda")))
    du0, dv0, dH0 = (x.cpu().numpy() for x in g._vec_to_fields(torch.as_tensor(d, device="cuda")))
    du, dv, dH = vanka_linear_update(st["u"], st["v"], st["H"], st["f_H"], ru, rv, rH, dH0, st["bed"], st["B"],
                                     st["beta"], st["gamma"], _params(), st["dx"], st["dt"], shift=0.0)
    got = [x.double().cpu().numpy() for x in g._vec_to_fields(d_t - d0)]
    tol = 1e-10 if precision == "fp64" else 2e-4
    for a, b in zip(got, (du, dv, dH)):
        assert _rel(a, 0.5 * b) <= tol
