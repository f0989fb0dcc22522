"""CPU checks of the FP64 oracle itself (no GPU).

These pin the oracle's internal consistency: the VJP is the transpose of the
JVP, the JVP is the derivative of the residual, the basal-friction gradient
is the beta-derivative of lambda . F, and the transfer operators reproduce
the reference formulas on hand-checkable inputs.  The reference-kernel
golden vectors are checked in test_golden.py.
"""
import numpy as np
import pytest

from conftest import random_state
from oracle import multigrid as O
from oracle import ssa
from oracle.ssa import Params
from oracle.vanka import local_cell_on, lu5_solve, vanka_deltas


def _args(st, p):
    return (st["bed"], st["B"], st["beta"], st["mask"], st["gamma"], p, st["dx"], st["dt"])


@pytest.mark.parametrize("gl,exact", [(False, False), (True, True)])
def test_vjp_is_transpose_of_jvp(gl, exact):
    st = random_state(n=16, seed=1)
    p = Params(gl_derivatives=gl)
    ju, jv, jH = ssa.jvp(st["u"], st["v"], st["H"], st["d_u"], st["d_v"], st["d_H"], *_args(st, p))
    lu, lv, lH = st["f_u"], st["f_v"], st["f_H"]
    vu, vv, vH = ssa.vjp(st["u"], st["v"], st["H"], lu, lv, lH, *_args(st, p), exact_boundary=exact)
    a = np.sum(lu * ju) + np.sum(lv * jv) + np.sum(lH * jH)
    b = np.sum(vu * st["d_u"]) + np.sum(vv * st["d_v"]) + np.sum(vH * st["d_H"])
    assert abs(a - b) <= 1e-12 * abs(a)


def test_reference_vjp_drops_boundary_terms_with_gl_derivatives():
    """The reference VJP is not the exact transpose when gl_derivatives is on
    (it drops clamped boundary reads); the oracle reproduces that."""
    st = random_state(n=16, seed=2)
    p = Params(gl_derivatives=True)
    ju, jv, jH = ssa.jvp(st["u"], st["v"], st["H"], st["d_u"], st["d_v"], st["d_H"], *_args(st, p))
    vu, vv, vH = ssa.vjp(st["u"], st["v"], st["H"], st["f_u"], st["f_v"], st["f_H"], *_args(st, p))
    a = np.sum(st["f_u"] * ju) + np.sum(st["f_v"] * jv) + np.sum(st["f_H"] * jH)
    b = np.sum(vu * st["d_u"]) + np.sum(vv * st["d_v"]) + np.sum(vH * st["d_H"])
    assert abs(a - b) > 1e-12 * abs(a)


def test_jvp_matches_central_differences():
    st = random_state(n=16, seed=3)
    p = Params(gl_derivatives=True)   # exact derivative only with the grounding-line terms on
    z = np.zeros_like
    F = lambda u, v, H: ssa.residual(u, v, H, z(u), z(v), z(H), *_args(st, p))
    eps = 1e-6
    Fp = F(st["u"] + eps * st["d_u"], st["v"] + eps * st["d_v"], st["H"] + eps * st["d_H"])
    Fm = F(st["u"] - eps * st["d_u"], st["v"] - eps * st["d_v"], st["H"] - eps * st["d_H"])
    J = ssa.jvp(st["u"], st["v"], st["H"], st["d_u"], st["d_v"], st["d_H"], *_args(st, p))
    for a, b, j in zip(Fp, Fm, J):
        fd = (a - b) / (2 * eps)
        assert np.linalg.norm(fd - j) <= 1e-6 * np.linalg.norm(j)


def test_grad_beta_exact_is_beta_derivative():
    st = random_state(n=12, seed=4)
    p = Params()
    lu, lv = st["f_u"], st["f_v"]
    g = ssa.grad_beta(st["u"], st["v"], st["H"], lu, lv, st["bed"], st["beta"], p, exact_boundary=True)
    rng = np.random.default_rng(5)
    d = rng.standard_normal(st["beta"].shape)
    z = np.zeros_like

    def L(beta):
        ru, rv, _ = ssa.residual(st["u"], st["v"], st["H"], z(st["u"]), z(st["v"]), z(st["H"]), st["bed"],
                                 st["B"], beta, st["mask"], st["gamma"], p, st["dx"], st["dt"])
        return np.sum(lu * ru) + np.sum(lv * rv)

    eps = 1e-4
    fd = (L(st["beta"] + eps * d) - L(st["beta"] - eps * d)) / (2 * eps)
    assert abs(fd - np.sum(g * d)) <= 1e-8 * abs(fd)


def test_grad_beta_reference_rule_differs_only_on_boundary():
    st = random_state(n=12, seed=6)
    p = Params()
    a = ssa.grad_beta(st["u"], st["v"], st["H"], st["f_u"], st["f_v"], st["bed"], st["beta"], p, False)
    b = ssa.grad_beta(st["u"], st["v"], st["H"], st["f_u"], st["f_v"], st["bed"], st["beta"], p, True)
    assert np.allclose(a[1:-1, 1:-1], b[1:-1, 1:-1], rtol=0, atol=1e-14)
    assert not np.allclose(a, b)


def test_lu5_matches_numpy_solve():
    rng = np.random.default_rng(7)
    A = rng.standard_normal((25, 10)) + 6 * np.eye(5).reshape(25, 1)
    b = rng.standard_normal((5, 10))
    x = np.array(lu5_solve(A, b))
    for k in range(10):
        assert np.allclose(A[:, k].reshape(5, 5) @ x[:, k], b[:, k], atol=1e-12)


def test_transfers_hand_values():
    uf = np.arange(4 * 5, dtype=float).reshape(4, 5)
    assert np.allclose(O.restrict_u(uf), 0.5 * (uf[0::2, 0::2] + uf[1::2, 0::2]))
    hf = np.arange(16, dtype=float).reshape(4, 4)
    assert np.allclose(O.restrict_cell(hf), [[2.5, 4.5], [10.5, 12.5]])
    assert np.allclose(O.restrict_max_pool(hf), [[5, 7], [13, 15]])
    # bilinear prolongation reproduces a field that is linear in the coarse coordinates (interior)
    yy, xx = np.mgrid[0:6, 0:6].astype(float)
    hc = 2 * yy + 3 * xx
    hfine = O.prolong_cell_bilinear(hc)
    jf = (np.arange(12) - 0.5) * 0.5
    want = 2 * jf[:, None] + 3 * jf[None, :]
    assert np.allclose(hfine[1:-1, 1:-1], want[1:-1, 1:-1])
    # injection and restriction are inverse on constants
    assert np.allclose(O.restrict_cell(O.prolong_cell_inject(hc)), hc)


def test_local_gating_rule():
    em = np.zeros((30, 30))
    assert not local_cell_on(em).any()
    em[14, 14] = 1.0   # first cell of block (1,1); also in the ring of blocks (0,0),(0,1),(1,0)
    on = local_cell_on(em)
    assert on[0:14, 0:14].all() and on[14:28, 14:28].all() and on[0:14, 14:28].all() and on[14:28, 0:14].all()
    assert not on[28:, :].any() and not on[:, 28:].any()


def test_vanka_fixed_point_of_a_solved_local_problem():
    """With f = F(U) the Vanka deltas vanish (U is a fixed point)."""
    st = random_state(n=16, seed=8)
    st["u"] *= 0.02
    st["v"] *= 0.02
    p = Params()
    z = np.zeros_like
    mask0 = np.zeros_like(st["H"])
    F = ssa.residual(st["u"], st["v"], st["H"], z(st["u"]), z(st["v"]), z(st["H"]), st["bed"], st["B"], st["beta"],
                     mask0, st["gamma"], p, st["dx"], st["dt"])
    du, dv, dH = vanka_deltas(st["u"], st["v"], st["H"], F[0], F[1], F[2], st["bed"], st["B"], st["beta"],
                              st["gamma"], p, st["dx"], st["dt"], 10)
    assert np.abs(du).max() < 1e-9 and np.abs(dv).max() < 1e-9 and np.abs(dH).max() < 1e-9


def test_pivoted_local_solve_matches_dense_solve():
    """lu5_solve_pivot (the reference's pivoted 5x5 solve) on random systems,
    one with a zero leading pivot where the unpivoted elimination breaks."""
    from oracle.vanka import lu5_solve, lu5_solve_pivot
    rng = np.random.default_rng(12)
    A = [rng.standard_normal(64) for _ in range(25)]
    b = [rng.standard_normal(64) for _ in range(5)]
    A[0][:8] = 0.0
    M = np.stack(A).reshape(5, 5, 64).transpose(2, 0, 1)
    ref = np.linalg.solve(M, np.stack(b).T[..., None])[..., 0]
    x = np.stack(lu5_solve_pivot(A, b)).T
    good = np.abs(np.linalg.det(M)) > 1e-3
    assert np.allclose(x[good], ref[good], rtol=1e-8, atol=1e-10)
    with np.errstate(divide="ignore", invalid="ignore"):
        xu = np.stack(lu5_solve(A, b)).T
    assert not np.isfinite(xu[:8]).all()


def test_oracle_check_relative_residuals():
    """The checker's |r| / |r0|: 1 for the starting state, the direct
    evaluation for another state, the same with worker processes."""
    from glide_b200.synthetic import dome_case
    from oracle.check import relative_residuals, residual_parts
    c = dome_case(2, n=32, dx=10000.0)
    rng = np.random.default_rng(5)
    state = (rng.standard_normal((32, 33)) * 20, rng.standard_normal((33, 32)) * 20, c.thickness + 3.0)
    geo = dict(bed=c.bed, B=c.B, beta=c.beta, H_prev=c.thickness, smb=c.smb, dx=c.dx, dt=c.dt, thklim=c.thklim)
    start = (np.zeros((32, 33)), np.zeros((33, 32)), c.thickness)
    r0 = np.sqrt(sum(residual_parts(*start, c.bed, c.B, c.beta, c.thickness, c.smb, c.dx, c.dt)))
    r1 = np.sqrt(sum(residual_parts(*state, c.bed, c.B, c.beta, c.thickness, c.smb, c.dx, c.dt)))
    serial = relative_residuals([(geo, [start, state])], workers=1)
    assert serial[0][0] == 1.0 and abs(serial[0][1] - r1 / r0) <= 1e-15 * r1 / r0
    par = relative_residuals([(geo, [state]), (geo, [start])], workers=2)
    assert par == [[serial[0][1]], [1.0]]
