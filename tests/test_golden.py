"""Pin the FP64 NumPy oracle to the reference's own CUDA kernels.

``tests/golden/reference_kernels_32.npz`` holds FP32 outputs of the reference
kernels (compiled from the reference tree, ``--use_fast_math``) on seeded
inputs, written by ``tests/golden/make_golden.py`` on a GPU box.  The oracle,
run in FP64 on the same (FP32-rounded) inputs, must agree within FP32
tolerances, stated per case below as norm-wise relative error:
  single operators (residual, JVP, VJP, grad)               <= 2e-6
  transfers                                                 <= 2e-7
  one Vanka sweep / local sweep / adjoint sweep pair        <= 1e-4
  one forward step (1 V-cycle, 3 levels, 200 coarse sweeps) <= 2e-5
  one adjoint V-cycle gradient                              <= 2e-5
(measured when the fixture was made: residual 4.5e-7, JVP/VJP <= 2.8e-7,
forward step 2.1e-6, adjoint gradient 2.1e-6)
"""
import os

import numpy as np
import pytest

from oracle import multigrid as O
from oracle import ssa
from oracle.ssa import Params
from oracle.vanka import local_cell_on, vanka_adjoint_color, vanka_deltas

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_kernels_32.npz")
pytestmark = pytest.mark.skipif(not os.path.exists(GOLD), reason="golden fixture not generated yet")


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k].astype(np.float64) for k in z.files}


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def _in(g, *names):
    return [g["in_" + n] for n in names]


def test_residual(gold):
    u, v, H, fu, fv, fH, bed, B, beta, mask, gamma = _in(gold, "u", "v", "H", "f_u", "f_v", "f_H", "bed", "B",
                                                          "beta", "mask", "gamma")
    r = ssa.residual(u, v, H, fu, fv, fH, bed, B, beta, mask, gamma, Params(), gold["dx"], gold["dt"])
    for a, k in zip(r, ("out_r_u", "out_r_v", "out_r_H")):
        assert rel(a, gold[k]) <= 2e-6


@pytest.mark.parametrize("gl", [0, 1])
def test_jvp_vjp(gold, gl):
    u, v, H, du, dv, dH, bed, B, beta, mask, gamma = _in(gold, "u", "v", "H", "d_u", "d_v", "d_H", "bed", "B",
                                                          "beta", "mask", "gamma")
    p = Params(gl_derivatives=bool(gl))
    j = ssa.jvp(u, v, H, du, dv, dH, bed, B, beta, mask, gamma, p, gold["dx"], gold["dt"])
    for a, k in zip(j, "uvH"):
        assert rel(a, gold[f"out_jvp{gl}_{k}"]) <= 2e-6
    fu, fv, fH = _in(gold, "f_u", "f_v", "f_H")
    l = ssa.vjp(u, v, H, fu, fv, fH, bed, B, beta, mask, gamma, p, gold["dx"], gold["dt"])
    for a, k in zip(l, "uvH"):
        assert rel(a, gold[f"out_vjp{gl}_{k}"]) <= 2e-6


def test_grad_beta(gold):
    u, v, H, du, dv, bed, beta = _in(gold, "u", "v", "H", "d_u", "d_v", "bed", "beta")
    g = ssa.grad_beta(u, v, H, du, dv, bed, beta, Params(), exact_boundary=False)
    assert rel(g, gold["out_grad_beta"]) <= 2e-6


@pytest.mark.parametrize("local", [False, True])
def test_vanka(gold, local):
    H, fu, fv, fH, bed, B, beta, gamma = _in(gold, "H", "f_u", "f_v", "f_H", "bed", "B", "beta", "gamma")
    u, v = gold["in_vanka_u"], gold["in_vanka_v"]
    on = local_cell_on(gold["in_error_mask"]) if local else None
    du, dv, dH = vanka_deltas(u, v, H, fu, fv, fH, bed, B, beta, gamma, Params(), gold["dx"], gold["dt"], 10, on)
    tag = "vlocal" if local else "vanka"
    # compare the updates U_new - U_old
    assert rel(0.5 * du, gold[f"out_{tag}_u"] - u) <= 1e-4
    assert rel(0.5 * dv, gold[f"out_{tag}_v"] - v) <= 1e-4
    assert rel(0.5 * dH, gold[f"out_{tag}_H"] - H) <= 1e-4


def test_vanka_adjoint(gold):
    u, v, H, bed, B, beta, mask, gamma = _in(gold, "u", "v", "H", "bed", "B", "beta", "mask", "gamma")
    lu, lv, lH = _in(gold, "d_u", "d_v", "d_H")
    fu, fv, fH = _in(gold, "f_u", "f_v", "f_H")
    p = Params()
    for color in (0, 1):
        vu, vv, vH = ssa.vjp(u, v, H, lu, lv, lH, bed, B, beta, mask, gamma, p, gold["dx"], gold["dt"])
        r = (fu - vu, fv - vv, fH - vH)
        lu, lv, lH = vanka_adjoint_color(lu, lv, lH, mask, r, u, v, H, bed, B, beta, gamma, p, gold["dx"],
                                         gold["dt"], color, 1.0)
    for a, k in zip((lu, lv, lH), "uvH"):
        assert rel(a, gold[f"out_vadj_{k}"]) <= 1e-4


def test_transfers(gold):
    t = gold
    assert rel(O.restrict_u(t["tr_uf"]), t["tr_restrict_u"]) <= 2e-7
    assert rel(O.restrict_v(t["tr_vf"]), t["tr_restrict_v"]) <= 2e-7
    assert rel(O.restrict_cell(t["tr_hf"]), t["tr_restrict_c"]) <= 2e-7
    assert rel(O.restrict_max_pool(t["tr_hf"]), t["tr_restrict_max"]) == 0.0
    assert rel(O.prolong_u_linear(t["tr_uc"]), t["tr_prolong_u_lin"]) <= 2e-7
    assert rel(O.prolong_u_bilinear(t["tr_uc"]), t["tr_prolong_u_bil"]) <= 2e-7
    assert rel(O.prolong_v_linear(t["tr_vc"]), t["tr_prolong_v_lin"]) <= 2e-7
    assert rel(O.prolong_v_bilinear(t["tr_vc"]), t["tr_prolong_v_bil"]) <= 2e-7
    assert rel(O.prolong_cell_inject(t["tr_hc"]), t["tr_prolong_c_inj"]) == 0.0
    assert rel(O.prolong_cell_bilinear(t["tr_hc"]), t["tr_prolong_c_bil"]) <= 2e-7


def test_forward_and_adjoint_step(gold):
    from glide_b200.synthetic import dome_case
    c = dome_case(0, n=32, dx=10000.0, n_levels=3)
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)
    ph = O.OracleIcePhysics(32, 32, c.dx, n_levels=3, thklim=c.thklim)
    ph.set_geometry(f32(c.bed), f32(c.thickness))
    ph.set_parameters(B=f32(c.B), beta=f32(c.beta), smb=f32(c.smb))
    u, v, H = ph.forward(c.dt, n_vcycles=1)
    assert rel(u, gold["step_u"]) <= 2e-5
    assert rel(v, gold["step_v"]) <= 2e-5
    assert rel(H, gold["step_H"]) <= 2e-5
    g = ph.adjoint(gold["step_dLu"], gold["step_dLv"], np.zeros((32, 32)), n_vcycles=1)
    assert rel(g, gold["step_grad_beta"]) <= 2e-5
