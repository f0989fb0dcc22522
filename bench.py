#!/usr/bin/env python
"""Benchmark: forward steps/s at 1e-6 relative residual, 1024x1024 SSA.

One step = one implicit forward time step (dt = 10 a) of a fresh seeded
1024x1024 ice-sheet geometry (dx = 1 km, 6 multigrid levels), solved until
|r|/|r0| <= tol (r combines r_u, r_v and FB(r_H, H - gamma); r0 is the
residual of the step's starting state u = v = 0, H = H_prev).  Synthetic
inputs stand in for the reference's datasets (no network here).

Arms
  (default)          this package on N GPUs, one process per GPU (replicas:
                     every rank solves its own geometries, no collective in the
                     data path; scaling "weak").  ``value`` is the fast path:
                     FP32 V-cycles with FP64 defect correction, full-step local
                     Newton (2 iterations) in the smoother, FP32/FP64
                     finishing sweeps with Anderson acceleration.  Beside it:
                     the same path started from the learned initial guess
                     (``learned_guess``), and the plain FP64 FAS path with the
                     reference's smoother (``plain_fp64_fas``), and both paths
                     on a time series started from the previous step's
                     solution (``warm_start``; the reference steps this way).
  --impl reference   the plain FAS algorithm in FP64 NumPy on the host cores
                     (the reference itself is GPU-only), timed on a bounded
                     sample: full-size fine-level Vanka sweeps, scaled to a
                     step by the plain path's cycle and sweep counts.

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "forward steps/s at 1e-6 rel. residual, 1024² SSA: plain FAS vs learned guess"
N = 1024
DX = 1000.0
LEVELS = 6
DT = 10.0
TOL = 1e-6
MAX_FINISH = 20000   # finishing-sweep budget of a step: every timed step must reach TOL


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--max-vcycles", type=int, default=40)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 FAS comparison arm")
    ap.add_argument("--no-guess", action="store_true", help="skip the learned-guess arm")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffers) measurement")
    ap.add_argument("--no-warm", action="store_true", help="skip the warm-start (time series) variant")
    ap.add_argument("--no-clocks", action="store_true", help="do not sample nvidia-smi clocks")
    ap.add_argument("--kernels", action="store_true",
                    help="per-kernel GB/s table on the marine configuration instead of the metric line")
    ap.add_argument("--kernels-n", type=int, default=4096, help="grid size of the --kernels table")
    ap.add_argument("--kernels-compare", action="store_true",
                    help="per-call times of the hot kernels at 1024^2 and 4096^2 (with --impl reference: the "
                         "reference's own kernels on the same state)")
    ap.add_argument("--guess-kernels", action="store_true",
                    help="tensor-core convolutions of the learned guess at 1024^2: per layer TFLOP/s and the "
                         "whole inference time")
    ap.add_argument("--eager", action="store_true",
                    help="launch kernels one by one instead of replaying CUDA graphs (for profiler runs)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--configs", action="store_true",
                    help="mixed vs FP64 on the 512^2 100-step and the 4096^2 20-step configurations (one JSON line)")
    ap.add_argument("--configs-only", default=None, help="with --configs: only the configuration named so")
    ap.add_argument("--configs-steps", type=int, default=0, help="with --configs: steps per series (0: 100 / 20)")
    ap.add_argument("--configs-iters", type=int, default=200, help="with --configs: L-BFGS iterations of the inversion")
    ap.add_argument("--configs-fd", type=int, default=16, help="with --configs: finite-difference directions")
    ap.add_argument("--configs-seconds", type=float, default=1200.0,
                    help="with --configs: wall time after which the inversion starts no new L-BFGS iteration")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampling (nvidia-smi) during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = sorted(float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        seen = set()
        for r in self.rows:
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    seen.add(name)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(seen),
                "samples": len(self.rows)}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The slowest rank's time: every rank solves its own geometries (replicas),
    so the job takes as long as its slowest rank."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seeds(rank, n):
    """Geometry seeds of one rank: disjoint between ranks, so N replicas solve
    N x n different geometries."""
    return [rank * 100_000 + k for k in range(n)]


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def tol_settings():
    """Plain FAS: the reference's smoother (10 local Newton iterations, step
    0.25, 10 local rounds) without the diagonal shift and with a small local
    threshold, so that the tolerance is reachable."""
    from glide_b200.solver import SolverSettings
    return SolverSettings(shift=0.0, err_threshold=1e-7)


def fast_settings():
    """Fast path: 2 full local Newton steps per cell, 2 local rounds, 6
    pre/post sweeps, 20 coarsest-level sweeps (the cycle and finishing-sweep
    counts on the benchmark geometries match those of 10 and 200)."""
    from glide_b200.solver import SolverSettings
    return SolverSettings(shift=0.0, err_threshold=1e-7, n_local_outer=2, n_newton=2, newton_step=1.0,
                          n_smooth=6, n_coarse=20)


FAST_KW = dict(finish_anderson=3, finish_fp32=True, finish_newton=2, finish_step=1.0, finish_linear="after",
               finish_fas_until=2e-4, finish_fas_patience=8,
               newton=True, newton_start=1e-2, newton_after=200, newton_min_gain=4.0, newton_local=2,
               newton_max_steps=6)
# the same-branch reference solves (TOL_TIGHT): the fast path's settings with the sweeps-only finish
TIGHT_KW = {k: v for k, v in FAST_KW.items() if not k.startswith("newton")}
# the fast path's smoother and finishing rule in FP64 (no FP32 correction stages; the
# Newton-Krylov finish on the FP64 hierarchy)
FP64_FAST_KW = dict(finish_anderson=3, finish_newton=2, finish_step=1.0,
                    **{k: v for k, v in FAST_KW.items() if k.startswith("newton")})
FAST_PATH = ("mixed FAS, full-step local Newton x2, finishing sweeps FP32 (FAS form, then linearised) / FP64 + "
             "Anderson(3); after 200 sweeps a Newton-Krylov finish (FGMRES, linear multigrid V-cycle "
             "preconditioner) while its steps gain >= 4x")


def make_cases(n, seeds):
    from glide_b200.synthetic import learned_guess_case
    return [learned_guess_case(seed=s, n=n, dx=DX * 1024 / n, n_levels=LEVELS) for s in seeds]


class Runner:
    """Solves fresh geometries with one IcePhysics instance."""

    def __init__(self, n, precision, guess_model=None, max_vcycles=40, settings=None, **kw):
        import torch
        from glide_b200 import IcePhysics
        self.ph = IcePhysics(n, n, DX * 1024 / n, n_levels=LEVELS, thklim=0.1, precision=precision,
                             settings=settings or tol_settings(), **kw)
        self.guess_model = guess_model
        self.max_vcycles = max_vcycles
        self.torch = torch

    def load_device(self, case):
        t = self.torch
        d = dict(bed=case.bed, H=case.thickness, B=case.B, beta=case.beta, smb=case.smb)
        return {k: t.as_tensor(v, dtype=self.ph.dtype, device="cuda") for k, v in d.items()}

    def step(self, dev, tol=None, max_finish_sweeps=MAX_FINISH):
        ph = self.ph
        ph.set_geometry(dev["bed"], dev["H"])
        ph.set_parameters(B=dev["B"], beta=dev["beta"], smb=dev["smb"])
        ph.reset_solution()
        guess = None
        if self.guess_model is not None:
            guess = self.guess_model.predict(dev["H"], dev["bed"], dev["beta"], dev["B"])
        ph.forward(DT, tol=TOL if tol is None else tol, max_vcycles=self.max_vcycles, guess=guess,
                   max_finish_sweeps=max_finish_sweeps)
        return dict(ph.last_info)

    def continue_step(self, dev, U, tol, max_finish_sweeps=MAX_FINISH):
        """Continue a solved step of the geometry ``dev`` from the state ``U``
        (a host or device FP64 vector) to ``tol``, relative to the residual of
        the step's starting state, with the finishing sweeps alone (no FAS
        cycle, which can carry a converged state onto another solution
        branch), so the answer stays on U's branch."""
        ph = self.ph
        ph.set_geometry(dev["bed"], dev["H"])
        ph.set_parameters(B=dev["B"], beta=dev["beta"], smb=dev["smb"])
        ph.reset_solution()
        ph._set_dt(DT)
        g = ph.grid
        g.f_H.copy_(g.H_prev / DT + g.smb)
        r0 = ph.residual_norm()
        g.U.copy_(U.to(device=g.U.device, dtype=g.U.dtype))
        ph.forward(DT, tol=tol, max_vcycles=0, max_finish_sweeps=max_finish_sweeps, r0=r0, update_geometry=False)
        return dict(ph.last_info)


def solution_error(sols, refs, n):
    """Largest relative 2-norm difference per field (u, v, H) between the
    states in ``sols`` and in ``refs`` (same geometries, same order)."""
    nu, nv = n * (n + 1), (n + 1) * n
    out = {"u": 0.0, "v": 0.0, "H": 0.0}
    for a, b in zip(sols, refs):
        for name, sl in (("u", slice(0, nu)), ("v", slice(nu, nu + nv)), ("H", slice(nu + nv, None))):
            d = float((a[sl] - b[sl]).norm() / b[sl].norm().clamp_min(1e-300))
            out[name] = max(out[name], d)
    return out


def flush_l2(buf):
    buf.add_(1.0)


def launches(runner):
    from glide_b200 import _native as N
    return N.load().glide_launch_count() + runner.ph.graph_launches


def time_steps(runner, devs, warmup, steps, world, flush, keep=None):
    """W untimed and K timed steps on fresh geometries.  Returns the total
    time, the per-step times (ms) and the solver records; with ``keep`` (a
    list) each timed step's FP64 state is copied to the host there, after its
    timed region."""
    import torch
    infos, step_ms = [], []
    for k in range(warmup):
        runner.step(devs[k % len(devs)])
    torch.cuda.synchronize()
    total = 0.0
    runner.launches = 0
    for k in range(steps):
        flush_l2(flush)
        barrier(world)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = launches(runner)
        a.record()
        infos.append(runner.step(devs[warmup + k]))
        b.record()
        torch.cuda.synchronize()
        runner.launches += launches(runner) - l0
        total += a.elapsed_time(b) / 1e3
        step_ms.append(round(a.elapsed_time(b), 2))
        if keep is not None:
            keep.append(runner.ph.grid.U.detach().to(torch.float64).cpu())
    return total, step_ms, infos


def host_inputs(cases):
    """Pinned FP64 host copies of every case's inputs (the end-to-end arm's source)."""
    import numpy as np
    import torch
    return [{k: torch.as_tensor(np.ascontiguousarray(v), dtype=torch.float64).pin_memory()
             for k, v in (("bed", c.bed), ("H", c.thickness), ("B", c.B), ("beta", c.beta), ("smb", c.smb))}
            for c in cases]


def e2e_step(ph, d, out_u, out_v, max_vcycles):
    """One step through the public API from host buffers: inputs copied to
    the device, the solve, (u, v) copied back."""
    dev = {key: val.to("cuda", non_blocking=True) for key, val in d.items()}
    ph.set_geometry(dev["bed"], dev["H"])
    ph.set_parameters(B=dev["B"], beta=dev["beta"], smb=dev["smb"])
    ph.reset_solution()
    u, v, H = ph.forward(DT, tol=TOL, max_vcycles=max_vcycles, max_finish_sweeps=MAX_FINISH)
    out_u.copy_(u, non_blocking=True)
    out_v.copy_(v, non_blocking=True)


def time_fast_and_e2e(fast, fdev, host, args, world, flush, n, keep=None):
    """The fast path timed two ways on the same geometries, step by step in
    alternation (so that both see the same clocks, warm state and sampler):
    ``value`` with inputs already resident in HBM, ``e2e`` through IcePhysics
    from pinned host buffers with the host<->device copies in its timed
    region.  Returns both totals, per-step times, solver records, launches
    and the bytes copied per e2e step."""
    import torch
    out_u = torch.empty((n, n + 1), dtype=torch.float64).pin_memory()
    out_v = torch.empty((n + 1, n), dtype=torch.float64).pin_memory()
    ph = fast.ph
    for k in range(args.warmup):
        fast.step(fdev[k])
        e2e_step(ph, host[k], out_u, out_v, args.max_vcycles)
    torch.cuda.synchronize()
    t_val = t_e2e = 0.0
    ms_val, ms_e2e, infos = [], [], []
    fast.launches = 0
    for k in range(args.steps):
        i = args.warmup + k
        for arm in ("value", "e2e"):
            flush_l2(flush)
            barrier(world)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = launches(fast)
            a.record()
            if arm == "value":
                infos.append(fast.step(fdev[i]))
            else:
                e2e_step(ph, host[i], out_u, out_v, args.max_vcycles)
            b.record()
            torch.cuda.synchronize()
            dt = a.elapsed_time(b)
            if arm == "value":
                fast.launches += launches(fast) - l0
                t_val += dt / 1e3
                ms_val.append(round(dt, 2))
                if keep is not None:
                    keep.append(ph.grid.U.detach().to(torch.float64).cpu())
            else:
                t_e2e += dt / 1e3
                ms_e2e.append(round(dt, 2))
    h2d = sum(t.numel() * t.element_size() for t in host[0].values())
    d2h = out_u.numel() * 8 + out_v.numel() * 8
    return t_val, t_e2e, ms_val, ms_e2e, infos, h2d, d2h


def kernel_timings(runner, launches=20):
    """Average launch durations (CUDA events on the launching stream) on the
    solved 1024^2 state of the fast path: the fine-level Vanka cell kernel in
    FP64 (the finishing sweeps) and FP32 (the V-cycle smoothing), with the
    fast path's local Newton settings, and the residual stencil in both."""
    import ctypes as C
    import torch
    from glide_b200 import _native as N
    ph = runner.ph
    lib = N.load()
    s = torch.cuda.current_stream()
    n_newton = ph.finish_newton if ph.finish_newton is not None else ph.settings.n_newton
    out = {}
    for g, tag in ((ph.grid, "64"), (ph.grid32, "32")):
        if g is None:
            continue
        a = g.level_args()
        saved = g.r.clone()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        for rep in range(2):  # first pass warms up
            torch.cuda.synchronize()
            ev[0].record(s)
            N.check(lib.glide_vanka_cells(C.byref(a), g.f_u.data_ptr(), g.f_v.data_ptr(), g.f_H.data_ptr(), launches,
                                          n_newton, float(ph.settings.shift), None, None, g._scratch.data_ptr(),
                                          s.cuda_stream), "vanka cells")
            ev[1].record(s)
            for _ in range(launches):
                g.compute_residual()
            ev[2].record(s)
            torch.cuda.synchronize()
        g.r.copy_(saved)
        out["cells" + tag] = ev[0].elapsed_time(ev[1]) / 1e3 / launches
        out["resid" + tag] = ev[1].elapsed_time(ev[2]) / 1e3 / launches
    return out


def roofline(t, n):
    """Roofline object of the dominant kernel (the FP32 Vanka cell kernel: the
    V-cycle smoothing and the FP32 finishing blocks, half of the fast path's
    kernel time) plus the FP64 cell kernel and the residual stencils."""
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    src = "measured" if "hbm_gbs" in peaks else "fallback"
    ncell = n * n
    scale = ncell / (1024 * 1024)
    def hbm_obj(bytes_per_cell, esz, sec):
        b = ncell * bytes_per_cell * esz
        return b / sec / 1e9
    fp64_peak = 148 * 64 * 2 * 1.965e9 / 1e12    # DFMA 64/clk/SM (ncu), nominal clock
    fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
    t64, t32 = t.get("cells64"), t["cells32"]
    ach = hbm_obj(VANKA_ARRAYS, 4, t32)
    roof = {"bound": "hbm", "kernel": "vanka_cells_kernel<float> (fine level, full sweep)",
            "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm, "peak_source": src,
            "traffic": VANKA32_DRAM_BYTES_1024 * scale,
            "traffic_source": "ncu dram__bytes_read+write, one 1024^2 launch",
            "algorithmic_bytes": ncell * VANKA_ARRAYS * 4, "launch_ms": t32 * 1e3,
            "limiter": "FP32 issue/latency (ncu at 1024^2: issue slots 61% active, 15 warps/SM at 128 registers, "
                       "1687 instructions per cell: FP32 930, integer 466, memory 129)",
            "alu": {"achieved_tflops": ncell * VANKA32_FLOPS_PER_CELL / t32 / 1e12, "peak_tflops": fp32_peak,
                    "frac": ncell * VANKA32_FLOPS_PER_CELL / t32 / 1e12 / fp32_peak,
                    "flops_per_cell": VANKA32_FLOPS_PER_CELL,
                    "peak_source": "nominal FP32 (148 SMs x 128 FFMA/clk)"}}
    if t64:
        roof["fp64_cells"] = {"kernel": "vanka_cells_kernel<double> (fine level, FP64 finishing blocks)",
                              "launch_ms": t64 * 1e3,
                              "achieved_tflops": ncell * VANKA64_FLOPS_PER_CELL / t64 / 1e12,
                              "frac_fp64_peak": ncell * VANKA64_FLOPS_PER_CELL / t64 / 1e12 / fp64_peak,
                              "hbm_frac": hbm_obj(VANKA_ARRAYS, 8, t64) / hbm}
    roof["stencil"] = {k: {"launch_ms": t[k] * 1e3, "achieved": hbm_obj(RESID_ARRAYS, e, t[k]),
                           "frac": hbm_obj(RESID_ARRAYS, e, t[k]) / hbm}
                       for k, e in (("resid64", 8), ("resid32", 4)) if k in t}
    return roof


def warm_start(runner, case, args, world, flush):
    """Steps/s of a time series on one geometry, each step started from the
    previous step's solution (the reference's way of stepping): W untimed and
    K timed consecutive steps, H_prev updated after each."""
    import torch
    ph = runner.ph
    dev = runner.load_device(case)
    ph.set_geometry(dev["bed"], dev["H"])
    ph.set_parameters(B=dev["B"], beta=dev["beta"], smb=dev["smb"])
    ph.reset_solution()
    tot, infos = 0.0, []
    for k in range(args.warmup + args.steps):
        flush_l2(flush)
        barrier(world)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ph.forward(DT, tol=TOL, max_vcycles=args.max_vcycles, max_finish_sweeps=MAX_FINISH)
        b.record()
        torch.cuda.synchronize()
        if k >= args.warmup:
            tot += a.elapsed_time(b) / 1e3
            infos.append(dict(ph.last_info))
    tot = max_over_ranks(tot, world)
    return {"value": world * args.steps / tot, "unit": "steps/s",
            "vcycles_per_step": [i.get("vcycles") for i in infos],
            "finish_sweeps_per_step": [i.get("finish_sweeps") for i in infos],
            "rel_residual_reached": [i.get("rel_residual") for i in infos],
            "series": f"steps {args.warmup + 1}..{args.warmup + args.steps} of one geometry, dt={DT:g} a"}


def branch_report(sols_a, sols_b, seeds, n, threshold=1e-3):
    """Geometries whose two answers differ by more than ``threshold``
    (relative 2-norm of u): where they differ (faces / cells whose value
    differs by more than ``threshold`` times the field's largest magnitude)."""
    nu, nv = n * (n + 1), (n + 1) * n
    out = []
    for a, b, seed in zip(sols_a, sols_b, seeds):
        du = float((a[:nu] - b[:nu]).norm() / b[:nu].norm().clamp_min(1e-300))
        if du <= threshold:
            continue
        rec = {"seed": seed, "u_rel": du}
        for name, sl in (("u", slice(0, nu)), ("v", slice(nu, nu + nv)), ("H", slice(nu + nv, None))):
            d = (a[sl] - b[sl]).abs()
            scale = float(b[sl].abs().max())
            rec[f"{name}_points_differing"] = int((d > threshold * scale).sum())
            rec[f"{name}_max_abs_diff"] = float(d.max())
        out.append(rec)
    return out


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args)
    n = args.n
    seeds = rank_seeds(rank, args.warmup + args.steps)
    cases = make_cases(n, seeds)
    timed_seeds = seeds[args.warmup:]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    guess_model = None
    try:
        from glide_b200.guess import load_default_model
        guess_model = load_default_model()
    except Exception as e:  # the learned-guess arm is reported as unavailable
        print(f"learned guess unavailable: {e}", file=sys.stderr)
    fast = Runner(n, "mixed", None, args.max_vcycles, fast_settings(), use_graphs=not args.eager, **FAST_KW)
    fdev = [fast.load_device(c) for c in cases]

    # the clock sampler runs over every timed arm
    sampler = ClockSampler(local)
    if not args.no_clocks:
        sampler.start()
    sols = {"fast": [], "learned_guess": [], "fp64_fast_smoother": [], "plain_fp64_fas": []}
    e2e_val, h2d, d2h, ms_e2e = None, 0, 0, []
    if args.no_e2e:
        t_fast, ms_fast, info_fast = time_steps(fast, fdev, args.warmup, args.steps, world, flush, sols["fast"])
    else:
        host = host_inputs(cases)
        t_fast, t_e2e, ms_fast, ms_e2e, info_fast, h2d, d2h = time_fast_and_e2e(fast, fdev, host, args, world,
                                                                                 flush, n, sols["fast"])
        e2e_val = world * args.steps / max_over_ranks(t_e2e, world)
        del host
    fast_launches = fast.launches
    t_fast = max_over_ranks(t_fast, world)
    value = world * args.steps / t_fast

    arms = {}
    if guess_model is not None and not args.no_guess:
        fast.guess_model = guess_model
        t, ms, infos = time_steps(fast, fdev, args.warmup, args.steps, world, flush, sols["learned_guess"])
        arms["learned_guess"] = (world * args.steps / max_over_ranks(t, world), ms, infos)
        fast.guess_model = None
    if not args.no_plain:
        # same smoother and finishing rule as the fast path, all in FP64: the precision gain alone
        f64 = Runner(n, "fp64", None, args.max_vcycles, fast_settings(), use_graphs=not args.eager, **FP64_FAST_KW)
        t, ms, infos = time_steps(f64, [f64.load_device(c) for c in cases], args.warmup, args.steps, world, flush,
                                  sols["fp64_fast_smoother"])
        arms["fp64_fast_smoother"] = (world * args.steps / max_over_ranks(t, world), ms, infos)
        del f64
        # the reference's smoother constants in FP64: the smoother gain on top
        plain = Runner(n, "fp64", None, args.max_vcycles, use_graphs=not args.eager)
        t, ms, infos = time_steps(plain, [plain.load_device(c) for c in cases], args.warmup, args.steps, world,
                                  flush, sols["plain_fp64_fas"])
        arms["plain_fp64_fas"] = (world * args.steps / max_over_ranks(t, world), ms, infos)
        del plain
        torch.cuda.empty_cache()
    sampler.stop()

    # accuracy of the fast path's answers: against the same solve continued to
    # TOL_TIGHT (its residual is evaluated in FP64, so that state solves the
    # FP64 discrete equations to TOL_TIGHT, on the same solution branch); it
    # continues from each fast answer with the finishing sweeps alone (the
    # Newton-Krylov finish is tuned for TOL and can stall short of TOL_TIGHT
    # at the non-smooth cells of the mass balance)
    tight = Runner(n, "mixed", None, args.max_vcycles, fast_settings(), use_graphs=not args.eager, **TIGHT_KW)
    sol_tight, rel_tight = [], []
    for k in range(args.steps):
        info = tight.continue_step(fdev[args.warmup + k], sols["fast"][k], TOL_TIGHT)
        rel_tight.append(info["rel_residual"])
        sol_tight.append(tight.ph.grid.U.detach().to(torch.float64).cpu())
    del tight
    torch.cuda.empty_cache()
    kept = [k for k, r in enumerate(rel_tight) if r is not None and r <= TOL_TIGHT]
    err = {"fast": solution_error([sols["fast"][k] for k in kept], [sol_tight[k] for k in kept], n) if kept else None,
           "reference_solution": f"the same solve continued to {TOL_TIGHT:g} relative residual (FP64 residual)",
           "reference_rel_residual": rel_tight,
           "reference_rel_residual_max": max(rel_tight[k] for k in kept) if kept else None,
           "dropped_seeds": [timed_seeds[k] for k in range(args.steps) if k not in kept],
           "note": "largest relative 2-norm difference per field over the timed steps whose reference reached "
                   f"{TOL_TIGHT:g}; dropped_seeds lists those that did not"}
    if kept:
        per = [solution_error([sols["fast"][k]], [sol_tight[k]], n)["u"] for k in kept]
        err["fast_u_per_seed"] = {str(timed_seeds[k]): e for k, e in zip(kept, per)}
        err["continuation_changed_branch"] = [timed_seeds[k] for k, e in zip(kept, per) if e > 1e-3]
    if sols["plain_fp64_fas"]:
        err["fast_vs_plain_fp64"] = solution_error(sols["fast"], sols["plain_fp64_fas"], n)
        if sols["learned_guess"]:
            err["learned_guess_vs_plain_fp64"] = solution_error(sols["learned_guess"], sols["plain_fp64_fas"], n)
        err["branches"] = branch_report(sols["fast"], sols["plain_fp64_fas"], timed_seeds, n)
        err["branches_note"] = ("geometries where the fast and plain answers differ by more than 1e-3 in u; "
                                "oracle_rel_residual shows both answers solve the FP64 equations to the tolerance")

    # end-of-run checks on rank 0 at N=1: the CPU baseline and the oracle's
    # FP64 residual of every arm's answers (the oracle as the checker, untimed)
    cpu, oracle_rel = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(cases[0], arms.get("plain_fp64_fas", (None, None, []))[2])
        oracle_rel = oracle_check(cases[args.warmup:], {**sols, "tight": sol_tight})
    del sols, sol_tight

    # dominant-kernel roofline (Vanka cell kernel, fine level of the FP32 hierarchy)
    roof = roofline(kernel_timings(fast), n)

    warm = None
    if not args.no_warm:
        warm = {"fast": warm_start(fast, cases[0], args, world, flush)}
        if not args.no_plain:
            plain_w = Runner(n, "fp64", None, args.max_vcycles, use_graphs=not args.eager)
            warm["plain_fp64_fas"] = warm_start(plain_w, cases[0], args, world, flush)
            del plain_w

    def arm(val, ms, infos, name):
        out = {"value": val, "unit": "steps/s", "step_ms": ms,
               "vcycles_per_step": [i.get("vcycles") for i in infos],
               "finish_sweeps_per_step": [i.get("finish_sweeps") for i in infos],
               "rel_residual_reached": [i.get("rel_residual") for i in infos]}
        if any("newton_steps" in i for i in infos):
            out["newton_steps_per_step"] = [i.get("newton_steps", 0) for i in infos]
            out["krylov_its_per_step"] = [i.get("krylov_its", 0) for i in infos]
        if oracle_rel is not None and name in oracle_rel:
            out["oracle_rel_residual"] = oracle_rel[name]
        return out

    if rank == 0:
        fast_arm = arm(value, ms_fast, info_fast, "fast")
        if oracle_rel is not None and "tight" in oracle_rel:
            err["reference_oracle_rel_residual"] = oracle_rel["tight"]
        summary = {"fast": value, "e2e": e2e_val}
        for name in ("learned_guess", "fp64_fast_smoother", "plain_fp64_fas"):
            summary[name] = arms[name][0] if name in arms else None
        if oracle_rel is not None:
            summary["oracle_rel_residual_max"] = {k: max(v) for k, v in oracle_rel.items() if v}
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_fast / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed: FP32 V-cycles, FP64 residual/norms)",
            "data": "synthetic (seeded grounded-dome geometries, fresh per step)",
            "config": {"workload": f"forward step to {TOL:g} rel. residual, {n}x{n}, dx={DX * 1024 / n:g} m, "
                                   f"{LEVELS} levels, dt={DT:g} a, fresh geometry per step",
                       "path": FAST_PATH, "seeds": timed_seeds,
                       "l2": "256 MB buffer written between timed steps", "parallelism": f"replicas x{world}"},
            **{k: v for k, v in fast_arm.items() if k not in ("value", "unit")},
            "learned_guess": (arm(*arms["learned_guess"], "learned_guess") if "learned_guess" in arms else
                              {"unavailable": "no trained model" if guess_model is None else "skipped"}),
            "fp64_fast_smoother": (arm(*arms["fp64_fast_smoother"], "fp64_fast_smoother")
                                   if "fp64_fast_smoother" in arms else None),
            "plain_fp64_fas": arm(*arms["plain_fp64_fas"], "plain_fp64_fas") if "plain_fp64_fas" in arms else None,
            "warm_start": warm,
            "error_vs_fp64": err,
            "e2e": {"value": e2e_val, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "step_ms": ms_e2e, "timing": "each e2e step timed right after the value step of the same "
                                                "geometry (alternating), same clock sampler"},
            "gpu_launches": fast_launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": sampler.summary(),
            "summary": summary,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def oracle_check(cases, sols, workers=None):
    """|r| / |r0| of every arm's answers, evaluated by the FP64 oracle on the
    host cores (the checker; after the timed regions)."""
    from oracle.check import relative_residuals
    names = [k for k, v in sols.items() if v]
    jobs = []
    for k, c in enumerate(cases):
        geo = dict(bed=c.bed, B=c.B, beta=c.beta, H_prev=c.thickness, smb=c.smb, dx=c.dx, dt=DT, thklim=c.thklim)
        states = []
        for name in names:
            U = sols[name][k].numpy()
            nu, nv = c.ny * (c.nx + 1), (c.ny + 1) * c.nx
            states.append((U[:nu].reshape(c.ny, c.nx + 1), U[nu:nu + nv].reshape(c.ny + 1, c.nx),
                           U[nu + nv:].reshape(c.ny, c.nx)))
        jobs.append((geo, states))
    rels = relative_residuals(jobs, workers=workers)
    return {name: [r[j] for r in rels] for j, name in enumerate(names)}


# Per-cell figures of the fine-level Vanka cell kernel with 2 local Newton
# iterations, from ncu op counts of one 1024^2 launch (dadd + dmul + 2 dfma,
# fadd + fmul + 2 ffma per cell), and its DRAM bytes per launch.
VANKA64_FLOPS_PER_CELL = 1611.0
VANKA32_FLOPS_PER_CELL = 1324.0
VANKA32_DRAM_BYTES_1024 = 43.98e6
# algorithmic arrays per cell: Vanka reads u, v, H, f_u, f_v, f_H, bed, B,
# beta, gamma and writes 5 delta arrays; the residual reads 11 and writes 3
VANKA_ARRAYS = 15
RESID_ARRAYS = 14


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 NumPy oracle on the host cores
# ---------------------------------------------------------------------------
def cpu_sweep_time(case, workers, repeats=1):
    import numpy as np
    from oracle.parallel import ParallelSweeper
    from oracle.ssa import Params
    ny, nx = case.ny, case.nx
    u = np.zeros((ny, nx + 1))
    v = np.zeros((ny + 1, nx))
    H = case.thickness.copy()
    f_u, f_v = np.zeros_like(u), np.zeros_like(v)
    f_H = H / DT + case.smb
    gamma = np.full_like(H, 0.1)
    ps = ParallelSweeper(workers)
    try:
        ps.deltas(u[:64], v[:65], H[:64], f_u[:64], f_v[:65], f_H[:64], case.bed[:64], case.B[:64],
                  case.beta[:64], gamma[:64], Params(), case.dx, DT, 10, shift=0.0)  # start the pool
        t = time.time()
        for _ in range(repeats):
            ps.deltas(u, v, H, f_u, f_v, f_H, case.bed, case.B, case.beta, gamma, Params(), case.dx, DT, 10,
                      shift=0.0)
        return (time.time() - t) / repeats
    finally:
        ps.close()


def sweeps_per_vcycle(levels=LEVELS, n_smooth=10, n_local_outer=10, n_local=10, n_coarse=200):
    """Fine-level-equivalent Vanka sweeps of one V-cycle with every local
    smoothing round active (the tolerance settings): sum over levels of
    sweeps x 4^-level."""
    w = 0.0
    for k in range(levels - 1):
        w += (2 * n_smooth + n_local_outer * n_local) * 4.0 ** (-k)
    w += n_coarse * 4.0 ** (-(levels - 1))
    return w


def plain_step_sweeps(infos):
    """Fine-level-equivalent sweeps of one plain FAS step: V-cycles x sweeps
    per V-cycle + finishing sweeps, averaged over the measured steps (fixed
    figures of an earlier GPU run of the plain arm when none are given)."""
    vc = [i.get("vcycles") or 0 for i in infos]
    fs = [i.get("finish_sweeps") or 0 for i in infos]
    if not vc:
        return REF_VCYCLES_PER_STEP, REF_FINISH_SWEEPS_PER_STEP
    return sum(vc) / len(vc), sum(fs) / len(fs)


def single_thread_sweep_time(case, rows=128):
    """One FP64 NumPy Vanka sweep over a rows-high strip of the grid in this
    process (one thread), scaled to the whole grid."""
    import numpy as np
    from oracle.ssa import Params
    from oracle.vanka import vanka_deltas
    nx = case.nx
    u = np.zeros((rows, nx + 1))
    v = np.zeros((rows + 1, nx))
    H = case.thickness[:rows].copy()
    t = time.time()
    vanka_deltas(u, v, H, np.zeros_like(u), np.zeros_like(v), H / DT + case.smb[:rows], case.bed[:rows],
                 case.B[:rows], case.beta[:rows], np.full_like(H, 0.1), Params(), case.dx, DT, 10, shift=0.0)
    return (time.time() - t) * case.ny / rows


def cpu_baseline(case, infos, workers=None):
    workers = workers or os.cpu_count() or 1
    t_sweep = cpu_sweep_time(case, workers)
    vpc, fin = plain_step_sweeps(infos)
    per_step = vpc * sweeps_per_vcycle() + fin
    t_step = per_step * t_sweep
    t1 = single_thread_sweep_time(case)
    return {"value": 1.0 / t_step, "unit": "steps/s", "cores": workers, "kind": "port", "modelled": True,
            "sample": f"one full-size {case.ny}x{case.nx} FP64 NumPy Vanka sweep ({t_sweep:.2f} s on {workers} "
                      f"processes), scaled by {vpc:.1f} V-cycles x {sweeps_per_vcycle():.1f} fine-equivalent "
                      f"sweeps + {fin:.0f} finishing sweeps per step (the plain FP64 arm's counts in this run)",
            "measured_s_per_sweep": t_sweep, "sweeps_per_step": per_step,
            "single_thread": {"value": 1.0 / (per_step * t1), "unit": "steps/s", "cores": 1,
                              "sample": f"one FP64 NumPy Vanka sweep over a 128-row strip in one process, "
                                        f"scaled to {case.ny} rows ({t1:.1f} s per sweep) and to a step as above"}}


TOL_TIGHT = 1e-8   # tolerance of the reference solutions of the accuracy check
# mean counts of the plain FP64 arm on this workload (GPU run of the default
# bench: the 20 timed fresh geometries, seeds 5-24)
REF_VCYCLES_PER_STEP = 3.15
REF_FINISH_SWEEPS_PER_STEP = 991.0


def run_reference(args):
    """The reference arm: the reference's algorithm (plain FAS, FP64, its
    smoother constants) in the FP64 NumPy oracle on the host cores.  A full
    1024^2 step takes tens of minutes on a CPU, so each timed step is a
    bounded sample -- one full-size fine-level Vanka sweep on that step's
    geometry -- and the steps/s is modelled from it with the plain arm's
    sweep counts; ``ms_per_step`` is the time actually measured per step."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    seeds = rank_seeds(0, args.warmup + args.steps)
    workers = os.cpu_count() or 1
    times = []
    for k in range(args.warmup + args.steps):
        case = make_cases(args.n, [seeds[k]])[0]
        t = cpu_sweep_time(case, workers)
        if k >= args.warmup:
            times.append(t)
    t_sweep = sum(times) / len(times)
    vpc, fin = plain_step_sweeps([])
    per_step = vpc * sweeps_per_vcycle() + fin
    t_step = per_step * t_sweep
    value = 1.0 / t_step
    sample = (f"per step: one full-size {args.n}x{args.n} FP64 NumPy Vanka sweep of that step's geometry on "
              f"{workers} processes ({t_sweep:.2f} s mean), scaled by {vpc:g} V-cycles x {sweeps_per_vcycle():.1f} "
              f"fine-equivalent sweeps + {fin:g} finishing sweeps per step")
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_sweep, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded grounded-dome geometries, fresh per step)",
            "config": {"workload": f"forward step to {TOL:g} rel. residual, {args.n}x{args.n}, dx={DX:g} m, "
                                   f"{LEVELS} levels, dt={DT:g} a, fresh geometry per step",
                       "seeds": seeds[args.warmup:], "parallelism": "host cores"},
            "impl": "reference",
            "modelled": {"value_is": "modelled from the measured sample", "measured_ms_per_step": 1e3 * t_sweep,
                         "modelled_ms_per_step": 1e3 * t_step, "fine_equivalent_sweeps_per_step": per_step,
                         "counts_source": "mean V-cycles and finishing sweeps of the plain FP64 GPU arm on these "
                                          "geometries (constants from its last measured run)"},
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": workers, "kind": "port", "modelled": True,
                             "sample": sample},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_series(case, precision, steps, cot_seed=7, arm="fast", newton=None):
    """``steps`` implicit steps of one geometry, each started from the
    previous one and solved to |r|/|r0| <= TOL, then the adjoint gradient of
    a seeded cotangent of (u, v) through the last step, solved to the same
    relative tolerance.  ``arm`` "fast": the fast path's solver (mixed, or
    the same solver in FP64); "plain": the plain FAS arm's settings.
    ``newton`` overrides the Newton-Krylov options.  Returns the final state,
    the gradient, the time of the steps and the relative residual each step
    reached."""
    import torch
    from glide_b200 import IcePhysics
    if arm == "plain":
        kw = dict(settings=tol_settings())
    else:
        kw = dict(settings=fast_settings(), **(FAST_KW if precision == "mixed" else FP64_FAST_KW))
        kw.update(newton or {})
    ph = IcePhysics(case.ny, case.nx, case.dx, n_levels=case.n_levels, thklim=case.thklim, precision=precision,
                    **kw, **case.kwargs)

    def start():
        ph.set_geometry(case.bed, case.thickness)
        ph.set_parameters(B=case.B, beta=case.beta, smb=case.smb)
        ph.reset_solution()

    start()
    ph.forward(case.dt, n_vcycles=1)  # warm-up: builds the per-cycle CUDA graphs
    start()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rels = []
    a.record()
    for _ in range(steps):
        ph.forward(case.dt, tol=TOL, max_vcycles=40, max_finish_sweeps=MAX_FINISH)
        rels.append(ph.last_info["rel_residual"])
    b.record()
    torch.cuda.synchronize()
    t = a.elapsed_time(b) / 1e3
    g = ph.grid
    state = [x.detach().to(torch.float64).clone() for x in (g.u, g.v, g.H)]
    gen = torch.Generator().manual_seed(cot_seed)
    cu = torch.randn(tuple(g.u.shape), generator=gen, dtype=torch.float64).to(g.u.device, g.dtype)
    cv = torch.randn(tuple(g.v.shape), generator=gen, dtype=torch.float64).to(g.u.device, g.dtype)
    # the adjoint linearises at the last step's state
    grad = ph.adjoint(cu, cv, torch.zeros_like(g.H), tol=TOL, max_vcycles=40,
                      max_finish_sweeps=MAX_FINISH).detach().to(torch.float64).clone()
    adj_rel = ph.last_adjoint_info.get("rel_residual")
    del ph
    torch.cuda.empty_cache()
    return state, grad, t, rels, adj_rel


def config_inversion(args, n=512, steps=50, every=10, iters=200, fd_dirs=16, eps=1e-6, seed=0, seconds=None):
    """Inversion of log beta on the plain-method dome at n x n (same domain:
    dx = 5 km * 64 / n): observations from a true log beta = log(1e3 Pa a/m)
    + a Gaussian random field (20 km correlation, sigma 1) after ``steps``
    implicit steps, with 2 % proportional Gaussian noise; the model runs the
    same steps checkpointed every ``every`` with recomputation (the
    hand-written VJP behind torch.autograd).  Misfit: the noise-weighted
    chi^2 / 2 per observation (sigma = 2 % of |u_obs| + 1 m/a).  Central
    differences on ``fd_dirs`` seeded directions (eps = 1e-6, FP64, steps
    and adjoints solved to 1e-10) against two gradients: the reference's
    adjoint (no grounding-line derivatives in the transposed Jacobian, 0.1 m
    active-set band) and the exact one (grounding-line derivatives, 1e-6 m
    band); the first four directions also at 2 eps (smoothness of the step
    map along them);
    L-BFGS-B for ``iters`` iterations or ``seconds`` of wall time (mixed
    precision, steps and adjoints to TOL, the exact adjoint) with Tikhonov
    weight 1e-3 on log beta."""
    import numpy as np
    import torch
    from glide_b200 import IcePhysics
    from glide_b200.adjoint import time_stepped
    from glide_b200.inverse import TimeSteppedObjective, finite_difference_check, invert_time_stepped
    from glide_b200.synthetic import _grf, beta_head, dome_case
    steps = args.configs_steps or steps
    c = dome_case(seed, n=n, dx=5000.0 * 64 / n, n_levels=5)
    rng = np.random.default_rng(seed + 1)
    logb_ref = float(np.log(beta_head(1e3)))
    logb_true = logb_ref + _grf(rng, n, n, c.dx, 20e3)

    def physics(precision, **extra):
        # the FP64 model of the finite differences is solved to 1e-10: sweeps-only finish
        kw = dict(settings=fast_settings(),
                  **(FAST_KW if precision == "mixed" else {k: v for k, v in FP64_FAST_KW.items()
                                                           if not k.startswith("newton")}))
        ph = IcePhysics(n, n, c.dx, n_levels=c.n_levels, thklim=c.thklim, precision=precision, **kw, **extra)
        ph.set_geometry(c.bed, c.thickness)
        ph.set_parameters(B=c.B, beta=np.exp(logb_true), smb=c.smb)
        return ph

    ph = physics("mixed", adjoint_exact_jacobian=True)
    ph.settings.adj_active_tol = 1e-6
    H0 = torch.as_tensor(c.thickness, device="cuda")
    t0 = time.time()
    with torch.no_grad():
        u, v, _ = time_stepped(torch.exp(torch.as_tensor(logb_true, device="cuda")), H0, ph, c.dt, steps, every,
                               1e-8, 1e-8, 60)
        u_obs = u * (1.0 + 0.02 * torch.randn(u.shape, generator=torch.Generator().manual_seed(5),
                                              dtype=u.dtype).to(u.device))
        v_obs = v * (1.0 + 0.02 * torch.randn(v.shape, generator=torch.Generator().manual_seed(6),
                                              dtype=v.dtype).to(v.device))
    t_obs = time.time() - t0
    sig_u = 0.02 * u.abs() + 1.0
    sig_v = 0.02 * v.abs() + 1.0
    wkw = dict(sigma_u=sig_u, sigma_v=sig_v, normalize=True)
    x0 = np.full(n * n, logb_ref)
    out = {"grid": f"{n}x{n}, dx={c.dx:g} m, {c.n_levels} levels, dt={c.dt:g} a", "steps": steps,
           "checkpoint_every": every, "observations_s": t_obs}
    # gradient check in FP64
    ph64 = physics("fp64")
    obj64 = TimeSteppedObjective(ph64, H0, u_obs, v_obs, c.dt, steps, every, reg_weight=1e-3, tol=1e-10,
                                 adj_tol=1e-10, **wkw)
    t0 = time.time()
    _, g_ref = obj64(x0)
    ph64x = physics("fp64", adjoint_exact_jacobian=True)
    ph64x.settings.adj_active_tol = 1e-6
    obj64x = TimeSteppedObjective(ph64x, H0, u_obs, v_obs, c.dt, steps, every, reg_weight=1e-3, tol=1e-10,
                                  adj_tol=1e-10, **wkw)
    _, g_exact = obj64x(x0)
    del obj64x, ph64x
    (e_ref, e_exact), pairs, smooth = finite_difference_check(obj64, x0, n_directions=fd_dirs, eps=eps,
                                                              grads=[g_ref, g_exact], smooth_dirs=min(4, fd_dirs))

    def stats(e):
        return {"rel_err": e, "max": max(e), "median": float(np.median(e))}
    out["fd_check"] = {"directions": fd_dirs, "eps": eps, "s": time.time() - t0,
                       "reference_adjoint": stats(e_ref), "exact_adjoint": stats(e_exact),
                       "fd_eps_vs_2eps_rel": smooth, "pairs_fd_ref_exact": pairs,
                       "max_step_rel_residual": obj64.max_step_rel, "tol": 1e-10,
                       "note": "reference_adjoint: J^T without grounding-line derivatives, active set H <= thklim "
                               "+ 0.1 m; exact_adjoint: with them, active set H <= thklim + 1e-6 m"}
    del obj64, ph64
    torch.cuda.empty_cache()
    # L-BFGS in mixed precision
    obj = TimeSteppedObjective(ph, H0, u_obs, v_obs, c.dt, steps, every, reg_weight=1e-3, tol=TOL, adj_tol=TOL,
                               **wkw)
    t0 = time.time()
    x, rec = invert_time_stepped(obj, x0, maxiter=iters, max_seconds=seconds)
    t_inv = time.time() - t0
    err0 = float(np.sqrt(np.mean((x0 - logb_true.ravel()) ** 2)))
    err1 = float(np.sqrt(np.mean((x - logb_true.ravel()) ** 2)))
    out["lbfgs"] = {**rec, "s": t_inv, "s_per_evaluation": t_inv / max(rec["evaluations"] - 1, 1),
                    "adjoint": "exact (grounding-line derivatives in J^T, 1e-6 m active-set band)",
                    "max_iterations": iters, "max_seconds": seconds,
                    "tol": TOL, "max_step_rel_residual": obj.max_step_rel,
                    "misfit_reduction": rec["final"]["misfit"] / rec["initial"]["misfit"],
                    "log_beta_rms_error": {"start": err0, "final": err1}}
    return out


def run_configs(args):
    """The 512^2 continental time series and the 4096^2 marine case, the
    fast mixed-precision path against plain FP64, every step and the final
    adjoint solved to TOL: throughput and relative difference of the final
    (u, v, H) and of the adjoint gradient."""
    from glide_b200.synthetic import ice_sheet_case, marine_case

    def rel(a, b):
        return float((a - b).norm() / b.norm().clamp_min(1e-300))

    out = {}
    # at 4096^2 the finishing sweeps converge too slowly to wait for: Newton-Krylov as soon as |r|/|r0| <= 1e-2
    nk_4096 = dict(newton_after=0, newton_min_gain=1.0, newton_max_steps=12)
    specs = [("c2_continental_512", ice_sheet_case(0, n=512, dx=1500.0, n_levels=5), args.configs_steps or 100, None),
             ("c5_marine_4096", marine_case(0, n=4096, dx=1000.0, n_levels=7), args.configs_steps or 20, nk_4096)]
    if not args.configs_only or "c3" in args.configs_only:
        out["c3_inversion_512"] = config_inversion(args, iters=args.configs_iters, fd_dirs=args.configs_fd,
                                                   seconds=args.configs_seconds)
    for name, case, steps, nk in specs:
        if args.configs_only and args.configs_only not in name:
            continue
        res = {}
        for prec in ("mixed", "fp64"):
            res[prec] = config_series(case, prec, steps, newton=nk)
        (sm, gm, tm, rm, am), (sd, gd, td, rd, ad) = res["mixed"], res["fp64"]
        out[name] = {
            "grid": f"{case.ny}x{case.nx}, dx={case.dx:g} m, {case.n_levels} levels, dt={case.dt:g} a",
            "steps": steps, "tol": TOL, "series": "each step started from the previous one",
            "fp64_arm": "the same solver in FP64 (fast smoother, Newton-Krylov on the FP64 hierarchy)",
            "newton": nk or {k: v for k, v in FAST_KW.items() if k.startswith("newton")},
            "mixed_steps_per_s": steps / tm, "fp64_steps_per_s": steps / td, "speedup": td / tm,
            "max_rel_residual": {"mixed": max(rm), "fp64": max(rd)},
            "adjoint_rel_residual": {"mixed": am, "fp64": ad},
            "rel_diff_vs_fp64": {"u": rel(sm[0], sd[0]), "v": rel(sm[1], sd[1]), "H": rel(sm[2], sd[2]),
                                 "grad_beta": rel(gm, gd)},
        }
    print(json.dumps({"configs": out}), flush=True)


# algorithmic arrays per cell of one launch (every distinct input read once,
# every output written once; u and v count as one cell array each)
KERNEL_ARRAYS = {"residual": 14, "jvp": 13, "vjp": 13, "grad_beta": 8, "vanka_cells": 15, "vanka_sweep": 26,
                 "norms": 5, "restrict_u": 1.25}


def kernel_table(args):
    """GB/s of every hot kernel on the marine configuration (4096^2 by default;
    all working sets far exceed the 126 MB L2), FP32 and FP64, CUDA events
    over 20 launches after a warm-up, against the measured copy bandwidth."""
    import ctypes as C
    import numpy as np
    import torch
    from glide_b200 import _native as N
    from glide_b200.grid import Grid
    from glide_b200.kernels import restrict_vfacet
    from glide_b200.synthetic import marine_case
    n = args.kernels_n
    case = marine_case(0, n=n, dx=1000.0 * 4096 / n, n_levels=7)
    lib = N.load()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    rng = np.random.default_rng(0)
    table = {}
    for dtype, tag in ((torch.float32, "fp32"), (torch.float64, "fp64")):
        g = Grid(n, n, case.dx, dt=DT, dtype=dtype)
        for k, val in (("H", case.thickness), ("H_prev", case.thickness), ("bed", case.bed), ("B", case.B),
                       ("beta", case.beta), ("smb", case.smb)):
            getattr(g, k).copy_(torch.as_tensor(val))
        g.gamma.fill_(0.1)
        g.u.copy_(torch.as_tensor(rng.standard_normal((n, n + 1)) * 100.0))
        g.v.copy_(torch.as_tensor(rng.standard_normal((n + 1, n)) * 100.0))
        g.f_H.copy_(g.H_prev / DT + g.smb)
        g.d_U.copy_(torch.as_tensor(rng.standard_normal(g.U.numel())))
        g.Lambda.copy_(torch.as_tensor(rng.standard_normal(g.U.numel())))
        grad = torch.empty_like(g.H)
        coarse = torch.empty((n // 2, n // 2 + 1), dtype=dtype, device="cuda")
        a = g.level_args()
        s = torch.cuda.current_stream()
        saved = g.U.clone()
        ops = {
            "residual": lambda: g.compute_residual(),
            "jvp": lambda: g.compute_jvp(),
            "vjp": lambda: g.compute_vjp(),
            "grad_beta": lambda: lib.glide_grad_beta(C.byref(a), g.lambda_u.data_ptr(), g.lambda_v.data_ptr(),
                                                      grad.data_ptr(), 0, s.cuda_stream),
            "vanka_cells": lambda: lib.glide_vanka_cells(C.byref(a), g.f_u.data_ptr(), g.f_v.data_ptr(),
                                                          g.f_H.data_ptr(), 1, 2, 0.0, None, None,
                                                          g._scratch.data_ptr(), s.cuda_stream),
            "vanka_sweep": lambda: g.vanka_sweep(1, n_inner=2, omega=0.5, shift=0.0, step=1.0),
            "norms": lambda: g.residual_norms(),
            "restrict_u": lambda: restrict_vfacet(g.u, u_coarse=coarse),
        }
        esz = 4 if dtype == torch.float32 else 8
        for name, fn in ops.items():
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(20):
                fn()
            e1.record(s)
            torch.cuda.synchronize()
            g.U.copy_(saved)
            t = e0.elapsed_time(e1) / 1e3 / 20
            gbs = KERNEL_ARRAYS[name] * esz * n * n / t / 1e9
            table.setdefault(name, {})[tag] = {"us": round(t * 1e6, 1), "GBs": round(gbs, 1),
                                               "frac": round(gbs / hbm, 3)}
        del g, saved
        torch.cuda.empty_cache()
    print(json.dumps({"kernels": table, "n": n, "case": "marine (floating shelves, beta = 0 there)",
                      "arrays_per_cell": KERNEL_ARRAYS, "peak_gbs": hbm,
                      "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                      "note": "vanka_* are ALU-bound (local 5x5 Newton per cell); GB/s shown for reference"}),
          flush=True)


def _kernel_state(n):
    """The kernel tables' inputs: the marine case at n x n with seeded random
    velocities (the same for both implementations)."""
    import numpy as np
    from glide_b200.synthetic import marine_case
    case = marine_case(0, n=n, dx=1000.0 * 4096 / n, n_levels=7)
    rng = np.random.default_rng(0)
    st = dict(H=case.thickness, bed=case.bed, B=case.B, beta=case.beta, f_H=case.thickness / DT + case.smb,
              u=rng.standard_normal((n, n + 1)) * 100.0, v=rng.standard_normal((n + 1, n)) * 100.0,
              d=rng.standard_normal(n * (n + 1) + (n + 1) * n + n * n))
    return case, st


def _time_ops(ops, reset=None, reps=20):
    import torch
    out = {}
    for name, fn in ops.items():
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        if reset is not None:
            reset()
        out[name] = round(e0.elapsed_time(e1) * 1e3 / reps, 1)
    return out


def kernel_compare_reference(args):
    """The reference's own CUDA kernels (glide/cuda/*.cu built from its sources
    into oracle/_ref, launched the way glide/grid.py launches them: FP32,
    16x16 blocks with stride 14, zero-fills before the atomics, the host-side
    axpy of a Vanka sweep) timed per call on the kernel tables' state, at
    1024^2 and 4096^2.  ``bench.py --kernels-compare`` times this package's
    kernels on the same state; profiles/ compares the two."""
    import torch
    from oracle import ref_replay as R
    res = {}
    for n in (1024, 4096):
        case, st = _kernel_state(n)
        g = R.RefGrid(n, n, case.dx, dt=DT)
        for k in ("H", "bed", "B", "beta", "f_H", "u", "v"):
            getattr(g, k).copy_(torch.as_tensor(st[k]))
        g.gamma.fill_(0.1)
        g.d_U.copy_(torch.as_tensor(st["d"]))
        g.Lambda.copy_(torch.as_tensor(st["d"]))
        saved = g.U.clone()
        ops = {"residual": g.compute_residual, "jvp": g.compute_jvp, "vjp": g.compute_vjp,
               "grad_beta": g.compute_grad_beta,
               "vanka_sweep_newton10": lambda: g.vanka_sweep(1, n_inner=10),
               "vanka_sweep_newton2": lambda: g.vanka_sweep(1, n_inner=2)}
        res[str(n)] = _time_ops(ops, reset=lambda: g.U.copy_(saved))
        del g
        torch.cuda.empty_cache()
    print(json.dumps({"impl": "reference", "kernels_us": res, "dtype": "f32",
                      "case": "marine (floating shelves), seeded random velocities",
                      "launch": "reference kernels built from the reference sources (sm_100a, --use_fast_math), "
                                "glide/grid.py's launch shape and host steps"}), flush=True)


def kernel_compare_ours(args):
    """This package's kernels on the state of kernel_compare_reference: FP32,
    the same operations (residual, JVP, VJP, grad_beta, one Vanka sweep with
    the reference's smoother constants at 10 and 2 local Newton iterations)."""
    import ctypes as C
    import torch
    from glide_b200 import _native as N
    from glide_b200.grid import Grid
    lib = N.load()
    res = {}
    for n in (1024, 4096):
        case, st = _kernel_state(n)
        g = Grid(n, n, case.dx, dt=DT, dtype=torch.float32)
        for k in ("H", "bed", "B", "beta", "f_H", "u", "v"):
            getattr(g, k).copy_(torch.as_tensor(st[k]))
        g.gamma.fill_(0.1)
        g.d_U.copy_(torch.as_tensor(st["d"]))
        g.Lambda.copy_(torch.as_tensor(st["d"]))
        grad = torch.empty_like(g.H)
        a = g.level_args()
        s = torch.cuda.current_stream().cuda_stream
        saved = g.U.clone()
        ops = {"residual": g.compute_residual, "jvp": g.compute_jvp, "vjp": g.compute_vjp,
               "grad_beta": lambda: lib.glide_grad_beta(C.byref(a), g.lambda_u.data_ptr(), g.lambda_v.data_ptr(),
                                                        grad.data_ptr(), 0, s),
               "vanka_sweep_newton10": lambda: g.vanka_sweep(1, n_inner=10, omega=0.5, shift=1.0, step=0.25),
               "vanka_sweep_newton2": lambda: g.vanka_sweep(1, n_inner=2, omega=0.5, shift=1.0, step=0.25)}
        res[str(n)] = _time_ops(ops, reset=lambda: g.U.copy_(saved))
        del g
        torch.cuda.empty_cache()
    print(json.dumps({"impl": "ours", "kernels_us": res, "dtype": "f32",
                      "case": "marine (floating shelves), seeded random velocities"}), flush=True)


def guess_kernel_table(args, n=1024, reps=20):
    """Every 3x3 convolution of the guess network at its shape for an n x n
    input (implicit-GEMM tcgen05 kernel, BF16 in, FP32 accumulate, bias +
    ReLU, BF16 out), CUDA events over ``reps`` launches after 3 warm-up
    launches; and one whole inference on a bench geometry.  TFLOP/s against
    the measured cuBLAS BF16 peak (burst)."""
    import torch
    from glide_b200 import guess as G
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    peak = float(peaks["bf16_tflops"])
    model = G.load_default_model()
    net = model.net
    side = []
    hw = n
    for lv in range(net.levels):
        side += [hw, hw]
        if lv < net.levels - 1:
            hw //= 2
    for lv in range(net.levels - 2, -1, -1):
        hw *= 2
        side += [hw, hw]

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps
    rows = []
    g = torch.Generator(device="cuda").manual_seed(0)
    with torch.no_grad():
        for (cin, cout), h in zip(net.plan, side):
            x = torch.randn(1, h, h, cin, generator=g, device="cuda").to(torch.bfloat16)
            W = (torch.randn(cout, 9 * cin, generator=g, device="cuda") * 0.05).to(torch.bfloat16)
            bias = torch.zeros(cout, device="cuda")
            y = torch.empty((h * h, cout), dtype=torch.bfloat16, device="cuda")
            ms = timed(lambda: G.conv3x3(x, W, y, bias=bias, relu=True, out_mode=1))
            fl = 2.0 * h * h * 9 * cin * cout
            rows.append({"hw": h, "cin": cin, "cout": cout, "us": round(ms * 1e3, 1),
                         "tflops": round(fl / ms / 1e9, 1), "frac_of_measured_bf16": round(fl / ms / 1e9 / peak, 4)})
        case = make_cases(n, [5])[0]
        dev = {k: torch.as_tensor(v, device="cuda") for k, v in (("H", case.thickness), ("bed", case.bed),
                                                                 ("beta", case.beta), ("B", case.B))}
        ms_inf = timed(lambda: model.predict(dev["H"], dev["bed"], dev["beta"], dev["B"]))
    print(json.dumps({"guess_kernels": rows, "inference_ms": round(ms_inf, 3),
                      "inference_gflop": round(net.flops(n, n) / 1e9, 1), "bf16_peak_tflops": peak,
                      "peak_source": "measured (cuBLAS bf16 8192^3, burst)"}), flush=True)


def main():
    args = parse()
    if args.impl == "reference" and args.kernels_compare:
        kernel_compare_reference(args)
    elif args.kernels_compare:
        kernel_compare_ours(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.kernels:
        kernel_table(args)
    elif args.guess_kernels:
        guess_kernel_table(args)
    elif args.configs:
        run_configs(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
