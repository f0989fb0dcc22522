"""The benchmark's answers judged by the FP64 oracle, at full size.

Four fresh 1024x1024 benchmark geometries (the bench's seeds 3-6; dx = 1 km,
6 levels, dt = 10 a) are solved by the fast mixed-precision path and by the
plain FP64 FAS path to |r|/|r0| <= 1e-6, and by the fast path continued to
1e-8 (the same-branch reference of the bench's accuracy figure).  Each answer's
relative residual is then evaluated by the FP64 NumPy oracle's own residual
(oracle/check.py: glide/physics.py:176-198 with the FB term of
glide/grid.py:205-208), independently of the GPU kernels that produced it:
<= 1.05e-6 for the tolerance solves, <= 1.05e-8 for the tight one (5 %
headroom for the difference between the GPU's and the oracle's FP64 rounding
of |r|).  Where the fast and plain answers differ by more than 1e-3 (relative
2-norm of u), both solving the FP64 equations to the tolerance shows that
the difference is a second solution of the discrete equations, not an error
of either path.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu

SEEDS = [3, 4, 5, 6]


def _u_rel(a, b, n):
    nu = n * (n + 1)
    return float((a[:nu] - b[:nu]).norm() / b[:nu].norm())


def test_bench_answers_solve_the_fp64_equations():
    import bench
    from oracle.check import relative_residuals
    n = 1024
    cases = bench.make_cases(n, SEEDS)
    fast = bench.Runner(n, "mixed", None, 40, bench.fast_settings(), **bench.FAST_KW)
    plain = bench.Runner(n, "fp64", None, 40)
    sols = {"fast": [], "plain": [], "tight": []}
    gpu_rel = {"fast": [], "plain": [], "tight": []}
    for c in cases:
        for name, runner, tol, sweeps in (("fast", fast, 1e-6, 4000), ("plain", plain, 1e-6, 4000),
                                          ("tight", fast, 1e-8, 20000)):
            info = runner.step(runner.load_device(c), tol=tol, max_finish_sweeps=sweeps)
            gpu_rel[name].append(info["rel_residual"])
            sols[name].append(runner.ph.grid.U.detach().to(torch.float64).cpu())
    jobs = []
    for k, c in enumerate(cases):
        geo = dict(bed=c.bed, B=c.B, beta=c.beta, H_prev=c.thickness, smb=c.smb, dx=c.dx, dt=bench.DT,
                   thklim=c.thklim)
        states = []
        for name in ("fast", "plain", "tight"):
            U = sols[name][k].numpy()
            nu, nv = n * (n + 1), (n + 1) * n
            states.append((U[:nu].reshape(n, n + 1), U[nu:nu + nv].reshape(n + 1, n), U[nu + nv:].reshape(n, n)))
        jobs.append((geo, states))
    orc = relative_residuals(jobs)
    report = []
    for k, seed in enumerate(SEEDS):
        r_fast, r_plain, r_tight = orc[k]
        branch = _u_rel(sols["fast"][k], sols["plain"][k], n)
        report.append((seed, r_fast, r_plain, r_tight, branch, gpu_rel["fast"][k], gpu_rel["plain"][k],
                       gpu_rel["tight"][k]))
        assert r_fast <= 1.05e-6, report
        assert r_plain <= 1.05e-6, report
        assert r_tight <= 1.05e-8, report
    print("seed, oracle |r|/|r0| fast / plain / tight, fast-vs-plain u, GPU fast / plain / tight:", report)
