"""Host-side helpers of bench.py (CPU): the roofline object, the accuracy
comparison of solutions and the plain arm's step counts."""
import math

import torch

import bench


def test_roofline_object_from_timings():
    t = {"cells32": 80e-6, "cells64": 170e-6, "resid32": 30e-6, "resid64": 62e-6}
    roof = bench.roofline(t, 1024)
    assert roof["bound"] == "hbm" and roof["unit"] == "GB/s"
    ncell = 1024 * 1024
    alg = ncell * bench.VANKA_ARRAYS * 4
    assert roof["algorithmic_bytes"] == alg
    assert math.isclose(roof["achieved"], alg / 80e-6 / 1e9)
    assert math.isclose(roof["frac"], roof["achieved"] / roof["peak"])
    assert math.isclose(roof["traffic"], bench.VANKA32_DRAM_BYTES_1024)
    assert math.isclose(roof["alu"]["achieved_tflops"], ncell * bench.VANKA32_FLOPS_PER_CELL / 80e-6 / 1e12)
    assert "fp64_cells" in roof and set(roof["stencil"]) == {"resid32", "resid64"}
    # a larger grid scales the measured traffic by its cell count
    assert math.isclose(bench.roofline(t, 2048)["traffic"], 4 * bench.VANKA32_DRAM_BYTES_1024)


def test_solution_error_per_field():
    n = 8
    nu, nv, nh = n * (n + 1), (n + 1) * n, n * n
    ref = torch.ones(nu + nv + nh, dtype=torch.float64)
    sol = ref.clone()
    sol[:nu] *= 1.01           # u off by 1 %
    sol[nu + nv:] *= 0.999     # H off by 0.1 %
    err = bench.solution_error([sol, ref.clone()], [ref, ref], n)
    assert math.isclose(err["u"], 0.01, rel_tol=1e-9)
    assert err["v"] == 0.0
    assert math.isclose(err["H"], 0.001, rel_tol=1e-9)


def test_plain_step_sweeps():
    assert bench.plain_step_sweeps([]) == (bench.REF_VCYCLES_PER_STEP, bench.REF_FINISH_SWEEPS_PER_STEP)
    infos = [{"vcycles": 2, "finish_sweeps": 100}, {"vcycles": 4, "finish_sweeps": 300}]
    assert bench.plain_step_sweeps(infos) == (3.0, 200.0)
