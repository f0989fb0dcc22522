"""Solver parity: whole V-cycles and forward/adjoint steps vs the FP64 oracle.

Tolerances: FP64 V-cycle state vs oracle <= 1e-8 relative (the cycle contains
branch points such as the active-set switch and the error-mask threshold, so
rounding-level differences of the operators can move a few values more than
in a single operator); FP32 path vs FP64 path <= 2e-3 relative after two
cycles of the reference settings.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _np(t):
    return t.detach().double().cpu().numpy()


def _case(n=32, levels=3):
    from glide_b200.synthetic import dome_case
    return dome_case(0, n=n, dx=5000.0 * 64 / n, n_levels=levels)


def _physics(c, precision, **kw):
    from glide_b200 import IcePhysics
    ph = IcePhysics(c.ny, c.nx, c.dx, n_levels=c.n_levels, thklim=c.thklim, precision=precision, **kw)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    return ph


def _oracle(c, **kw):
    from oracle.multigrid import OracleIcePhysics
    ph = OracleIcePhysics(c.ny, c.nx, c.dx, n_levels=c.n_levels, thklim=c.thklim, **kw)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    return ph


def test_forward_fp64_vs_oracle():
    c = _case()
    ph = _physics(c, "fp64", use_graphs=False)
    u, v, H = ph.forward(c.dt, n_vcycles=1)
    ou, ov, oH = _oracle(c).forward(c.dt, n_vcycles=1)
    assert _rel(_np(u), ou) <= 1e-8
    assert _rel(_np(v), ov) <= 1e-8
    assert _rel(_np(H), oH) <= 1e-8


def test_forward_graph_matches_eager():
    c = _case()
    a = _physics(c, "fp64", use_graphs=False)
    b = _physics(c, "fp64", use_graphs=True)
    for _ in range(2):
        ua, va, Ha = a.forward(c.dt, n_vcycles=2)
        ub, vb, Hb = b.forward(c.dt, n_vcycles=2)
    assert np.array_equal(_np(ua), _np(ub)) and np.array_equal(_np(Ha), _np(Hb))


def test_forward_fp32_close_to_fp64():
    c = _case()
    a = _physics(c, "fp64")
    b = _physics(c, "fp32")
    ua, va, Ha = a.forward(c.dt, n_vcycles=2)
    ub, vb, Hb = b.forward(c.dt, n_vcycles=2)
    assert _rel(_np(ub), _np(ua)) <= 2e-3
    assert _rel(_np(Hb), _np(Ha)) <= 2e-3


def test_adjoint_fp64_vs_oracle():
    c = _case()
    ph = _physics(c, "fp64", use_graphs=False)
    orc = _oracle(c)
    ph.forward(c.dt, n_vcycles=1)
    orc.forward(c.dt, n_vcycles=1)
    rng = np.random.default_rng(3)
    dLu = rng.standard_normal((c.ny, c.nx + 1)) * 1e-3
    dLv = rng.standard_normal((c.ny + 1, c.nx)) * 1e-3
    dLH = np.zeros((c.ny, c.nx))
    g = ph.adjoint(dLu, dLv, dLH, n_vcycles=1)
    og = orc.adjoint(dLu, dLv, dLH, n_vcycles=1)
    assert _rel(_np(g), og) <= 1e-8


@pytest.mark.parametrize("mode", [True, "after"])
def test_mixed_linear_finish_goes_below_the_fp32_correction_floor(mode):
    """Mixed precision with the linear defect-correction finish (from the
    start, or after the FAS-form FP32 blocks) reaches |r|/|r0| <= 1e-9
    (measured by the FP64 oracle's own residual) with FP32 finishing blocks
    only; the FAS-form FP32 correction floors near eps32 times the size of the
    operator's terms."""
    from glide_b200 import IcePhysics, SolverSettings
    from oracle.multigrid import OracleIcePhysics, residual_norm
    c = _case(n=64, levels=3)
    st = SolverSettings(shift=0.0, err_threshold=1e-7, n_local_outer=2, n_newton=2, newton_step=1.0)
    ph = IcePhysics(c.ny, c.nx, c.dx, n_levels=c.n_levels, thklim=c.thklim, precision="mixed", settings=st,
                    finish_fp32=True, finish_linear=mode, finish_anderson=3)
    ph.set_geometry(c.bed, c.thickness)
    ph.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    u, v, H = ph.forward(c.dt, tol=1e-9, update_geometry=False, max_vcycles=1)
    info = ph.last_info
    assert info["rel_residual"] <= 1e-9
    assert info["finish_blocks"]["fp64"] == 0 and info["finish_blocks"]["fp32"] > 0, info
    orc = OracleIcePhysics(c.ny, c.nx, c.dx, n_levels=c.n_levels, thklim=c.thklim)
    orc.set_geometry(c.bed, c.thickness)
    orc.set_parameters(B=c.B, beta=c.beta, smb=c.smb)
    g = orc.grid
    g.dt = c.dt
    g.f_H = g.H_prev / g.dt + g.smb
    r0 = residual_norm(g)
    g.u, g.v, g.H = _np(u), _np(v), _np(H)
    assert residual_norm(g) / r0 <= 1.2e-9


def test_fast_path_reaches_tolerance_on_benchmark_geometries():
    """The benchmark's fast path (mixed precision, FAS-form then linearised
    FP32 finishing blocks, Anderson extrapolation, FP64 hand-over) reaches
    |r|/|r0| <= 1e-6 on twelve fresh 1024^2 geometries and on a warm-started
    series.  Seed 9's first V-cycle diverges and is undone; seed 11 needs the
    FAS form kept through slow, uneven blocks; seed 1's answer is also checked
    with the FP64 oracle's own residual."""
    import torch
    import bench
    from oracle.multigrid import OracleIcePhysics, residual_norm
    seeds = list(range(12))
    cases = bench.make_cases(1024, seeds)
    run = bench.Runner(1024, "mixed", settings=bench.fast_settings(), **bench.FAST_KW)
    for seed, case in zip(seeds, cases):
        info = run.step(run.load_device(case))
        assert info["rel_residual"] <= bench.TOL, (seed, info)
        if seed == 1:
            ph = run.ph
            orc = OracleIcePhysics(case.ny, case.nx, case.dx, n_levels=1, thklim=0.1)
            orc.set_geometry(case.bed, case.thickness)
            orc.set_parameters(B=case.B, beta=case.beta, smb=case.smb)
            g = orc.grid
            g.dt = bench.DT
            g.f_H = g.H_prev / g.dt + g.smb
            r0 = residual_norm(g)
            g.u, g.v, g.H = _np(ph.grid.u), _np(ph.grid.v), _np(ph.grid.H)
            assert residual_norm(g) / r0 <= 1.05 * bench.TOL
    ph = run.ph
    dev = run.load_device(cases[0])
    ph.set_geometry(dev["bed"], dev["H"])
    ph.set_parameters(B=dev["B"], beta=dev["beta"], smb=dev["smb"])
    ph.reset_solution()
    for step in range(6):
        ph.forward(bench.DT, tol=bench.TOL, max_vcycles=40)
        assert ph.last_info["rel_residual"] <= bench.TOL, (step, ph.last_info)
    torch.cuda.synchronize()
