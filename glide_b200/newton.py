"""Newton-Krylov finishing solver of the mixed-precision tolerance solve.

No counterpart in the reference: glide/physics.py:141-209 runs a fixed number
of FAS V-cycles and never solves to a tolerance.  Once the FAS phase of
``IcePhysics.forward(tol=...)`` has brought |r|/|r0| below
``newton_start``, each Newton step

1. evaluates r = F(U) - f in FP64 (the residual the tolerance is measured
   on); cells with H - dt r_H <= gamma (the Vanka smoother's rule) form the
   active set, whose rows become the constraint H - gamma
   (``glide_newton_rhs``);
2. solves J(fl32 U) d = -r in FP32 (or J(U) d = -r in FP64 on the FP64
   path) with FGMRES(m) to a relative tolerance,
   right-preconditioned by one linear multigrid V-cycle per iteration
   (``glide_linear_vcycle``, replayed from a CUDA graph): linear Vanka sweeps
   on every level with the local matrices factored once per step, each coarse
   level linearised at the restricted state.  J includes the grounding-line
   derivatives, so that it is the Jacobian of the residual (they do not
   change the residual itself).  Gram-Schmidt runs twice per iteration with
   FP64 dot products (``glide_dots``/``glide_combine``);
3. sets U += alpha fl64(d) with H >= gamma, halving alpha until |r| falls.

In the mixed path the FP32 correction's rounding error scales with d, not
with the operator's terms, so the steps converge to the FP64 solution
(iterative refinement).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _native as N


class NewtonKrylov:
    """The Newton-Krylov finish of one IcePhysics object.  With
    ``precision="mixed"`` the linear solves run on the FP32 hierarchy (FP32
    corrections of the FP64 state); with ``precision="fp64"`` on the FP64
    hierarchy itself (level 0's state is then the state being corrected)."""

    def __init__(self, physics, m=20):
        self.ph = physics
        self.lib = N.load()
        self.mixed = physics.grid32 is not None
        self.gs = physics.grids32 if self.mixed else physics.grids
        g0 = self.gs[0]
        self.n = g0.nb * g0.n_total
        self.m = int(m)
        dev = g0.device
        self.dtype, self.code = g0.dtype, g0.code
        self.V = torch.zeros(self.m + 1, self.n, dtype=self.dtype, device=dev)
        self.Z = torch.zeros(self.m, self.n, dtype=self.dtype, device=dev)
        self.w = torch.zeros(self.n, dtype=self.dtype, device=dev)
        self.x = torch.zeros(self.n, dtype=self.dtype, device=dev)
        self.hb = torch.zeros(2 * self.m + 4, dtype=torch.float64, device=dev)
        self.y = torch.zeros(self.m, dtype=torch.float64, device=dev)
        self.parts = torch.zeros(self.lib.glide_dots_parts(self.n) * 32, dtype=torch.float64, device=dev)
        self.base = torch.empty_like(physics.grid.U)
        self._levels = {}
        self._graphs = {}
        for g in self.gs:
            g.newton_buffers()

    # ------------------------------------------------------------------ plumbing
    def _s(self):
        return N.stream_handle()

    def levels(self):
        """Level array (rebuilt per dt: the level descriptors carry dt)."""
        key = float(self.gs[0].dt)
        if key not in self._levels:
            arr = (N.Level * len(self.gs))()
            for k, g in enumerate(self.gs):
                arr[k] = g.newton_level(self.ph.gl_sigmoid_c)
            self._levels[key] = arr
        return self._levels[key], len(self.gs)

    def graph(self, cfg):
        key = float(self.gs[0].dt)
        if key not in self._graphs:
            arr, n = self.levels()
            h = C.c_void_p()
            c0 = self.lib.glide_launch_count()
            N.check(self.lib.glide_graph_create(arr, n, C.byref(cfg), 2, C.byref(h)), "linear V-cycle graph")
            self._graphs[key] = (h, self.lib.glide_launch_count() - c0)
        return self._graphs[key]

    def _replay(self, cfg):
        """One linear V-cycle from its graph; the kernels it runs are added to
        the physics object's ``graph_launches`` (the library's counter sees
        captured launches once, at capture)."""
        h, nodes = self.graph(cfg)
        N.check(self.lib.glide_graph_launch(h, self._s()), "linear V-cycle")
        self.ph.graph_launches += nodes

    def release(self):
        for h, _ in self._graphs.values():
            self.lib.glide_graph_destroy(h)
        self._graphs.clear()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def _dots(self, V, k, w, out):
        N.check(self.lib.glide_dots(self.code, self.n, k, V.data_ptr(), self.n, w.data_ptr(), out.data_ptr(),
                                    self.parts.data_ptr(), self._s()), "dots")

    def _combine(self, V, k, coef, alpha, out, beta):
        N.check(self.lib.glide_combine(self.code, self.n, k, V.data_ptr(), self.n, coef.data_ptr(), float(alpha),
                                       out.data_ptr(), float(beta), self._s()), "combine")

    def _scale(self, out, x, a):
        N.check(self.lib.glide_lincomb(self.code, out.data_ptr(), x.data_ptr(), float(a), None, 0.0, self.n, self._s()),
                "lincomb")

    # ------------------------------------------------------------------ FGMRES
    def fgmres(self, cfg, rtol):
        """x ~ J^-1 (-g) for g = level 0's lin_rhs; returns (iterations, relative residual estimate)."""
        lib, m = self.lib, self.m
        g0 = self.gs[0]
        buf = g0.newton_buffers()
        rhs, d = buf["lin_rhs"], buf["lin_d"]
        a0 = self.levels()[0][0].a
        hb = self.hb
        self._dots(rhs, 1, rhs, hb[:1])
        beta = math.sqrt(float(hb[0].item()))
        self.x.zero_()
        if not (beta > 0.0 and math.isfinite(beta)):
            return 0, 0.0 if beta == 0.0 else float("nan")
        self._scale(self.V[0], rhs, -1.0 / beta)
        Hm = np.zeros((m + 1, m))
        y = None
        res = 1.0
        its = 0
        wu, wv, wH = g0._vec_to_fields(self.w)
        for j in range(m):
            self._scale(rhs, self.V[j], -1.0)            # V-cycle solves J z = -rhs = V[j]
            self._replay(cfg)
            self.Z[j].copy_(d)
            zu, zv, zH = g0._vec_to_fields(self.Z[j])
            N.check(lib.glide_jvp(C.byref(a0), zu.data_ptr(), zv.data_ptr(), zH.data_ptr(), wu.data_ptr(),
                                  wv.data_ptr(), wH.data_ptr(), self._s()), "jvp")
            k = j + 1
            h1, h2, hn = hb[:k], hb[m + 1:m + 1 + k], hb[2 * m + 2:2 * m + 3]
            self._dots(self.V, k, self.w, h1)
            self._combine(self.V, k, h1, -1.0, self.w, 1.0)
            self._dots(self.V, k, self.w, h2)             # second pass (CGS2)
            self._combine(self.V, k, h2, -1.0, self.w, 1.0)
            self._dots(self.w, 1, self.w, hn)
            h = hb.cpu().numpy()
            Hm[:k, j] = h[:k] + h[m + 1:m + 1 + k]
            hnorm = math.sqrt(max(h[2 * m + 2], 0.0))
            Hm[k, j] = hnorm
            its = k
            e1 = np.zeros(k + 1)
            e1[0] = beta
            y, *_ = np.linalg.lstsq(Hm[:k + 1, :k], e1, rcond=None)
            res = float(np.linalg.norm(e1 - Hm[:k + 1, :k] @ y)) / beta
            if not (np.isfinite(res) and np.all(np.isfinite(y))):
                return its, float("nan")
            if res <= rtol or hnorm <= 1e-30 * beta:
                break
            if j + 1 < m:
                self._scale(self.V[j + 1], self.w, 1.0 / hnorm)
        self.y[:its].copy_(torch.as_tensor(y, dtype=torch.float64))
        self._combine(self.Z, its, self.y, 1.0, self.x, 0.0)
        return its, res

    # ------------------------------------------------------------------ Newton
    def local_sweeps(self, r0, rel, rounds=2, sweeps=5):
        """Error-gated FP64 Vanka sweeps after a Newton step: the residual a
        step leaves is concentrated in a few cells where the residual is not
        smooth (the max() of the floating surface, the upwind switch), which
        the local nonlinear solves resolve.  Tiles whose error indicator
        exceeds 5x the residual's RMS are swept.  Kept only if |r| falls."""
        ph, g64, lib = self.ph, self.ph.grid, self.lib
        s = self._s()
        keep = self.base
        keep.copy_(g64.U)
        g64.gamma.fill_(ph.thklim)
        a = g64.level_args()
        n_pts = g64.nb * g64.n_total
        for _ in range(rounds):
            g64.compute_residual()
            rms = math.sqrt(float(g64.residual_norms().sum().item()) / n_pts)
            N.check(lib.glide_error_mask(C.byref(a), g64.r_u.data_ptr(), g64.r_v.data_ptr(), g64.r_H.data_ptr(),
                                         5.0 * rms, g64.error_mask.data_ptr(), g64._flags.data_ptr(),
                                         g64._any_active.data_ptr(), s), "error mask")
            g64._sweeps(sweeps, 2, ph.settings.omega, ph.settings.shift, True, 1.0)
        new = ph.residual_norm() / r0
        if math.isfinite(new) and new < rel:
            return new
        g64.U.copy_(keep)
        return rel

    def solve(self, r0, tol, rel, hist, info, max_steps=10, rtol=1e-2, max_ls=6, min_gain=1.0, local_rounds=0):
        """Newton steps from the current FP64 state until |r|/|r0| <= tol, no
        step reduces |r|, or a step gains less than ``min_gain``x (then the
        caller's sweeps take over).  ``local_rounds`` > 0 follows each step by
        error-gated FP64 sweeps (``local_sweeps``).  Returns the relative
        residual reached."""
        ph = self.ph
        lib = self.lib
        g64 = ph.grid
        g0 = self.gs[0]
        s = self._s()
        cfg = ph.settings.native(ph.thklim)
        arr, nlev = self.levels()
        buf = g0.newton_buffers()
        a64 = g64.level_args()
        ntot = g64.nb * g64.n_total
        steps = its_total = 0
        while steps < max_steps and rel > tol:
            g64.gamma.fill_(ph.thklim)
            g64.compute_residual()
            N.check(lib.glide_newton_rhs(C.byref(a64), g64.r.data_ptr(), buf["lin_rhs"].data_ptr(),
                                         buf["r_raw"].data_ptr(), buf["mask"].data_ptr(), self.code, s), "newton rhs")
            if self.mixed:
                N.check(lib.glide_convert(N.F32, g0.U.data_ptr(), g64.U.data_ptr(), ntot, 0, s), "convert")
            N.check(lib.glide_linear_setup(arr, nlev, C.byref(cfg), s), "linear setup")
            # forcing term: no more accuracy than the step needs (Newton converges fast here)
            eta = min(0.5, max(rtol, 0.3 * tol / rel))
            its, lres = self.fgmres(cfg, eta)
            its_total += its
            if not math.isfinite(lres):
                break
            self.base.copy_(g64.U)
            alpha, accepted = 1.0, False
            for _ in range(max_ls):
                N.check(lib.glide_newton_update(C.byref(a64), g64.U.data_ptr(), self.base.data_ptr(),
                                                self.x.data_ptr(), self.code, alpha, s), "newton update")
                new = ph.residual_norm() / r0
                if math.isfinite(new) and new < rel:
                    accepted = True
                    break
                alpha *= 0.5
            if not accepted:
                g64.U.copy_(self.base)
                info["newton_rejected"] = info.get("newton_rejected", 0) + 1
                break
            if local_rounds > 0 and new > tol:
                new = self.local_sweeps(r0, new, rounds=local_rounds)
            gain = rel / new
            rel = new
            hist.append(rel)
            steps += 1
            if gain < min_gain:
                info["newton_slow"] = info.get("newton_slow", 0) + 1
                break
        info["newton_steps"] = info.get("newton_steps", 0) + steps
        info["krylov_its"] = info.get("krylov_its", 0) + its_total
        return rel


class AdjointKrylov:
    """FGMRES(m) for the adjoint system of a solved step,

        J_m(U)^T lam = f_adj,

    J_m: the Jacobian of F(U) - f with the rows of the active cells
    (H <= gamma + adj_active_tol) replaced by the identity, the system the
    reference's adjoint V-cycle relaxes (glide/solver.py:160-220,
    glide/grid.py:319-334).  Right-preconditioned by one adjoint V-cycle per
    iteration (``glide_adjoint_vcycle`` from lam = 0, replayed from a CUDA
    graph; on the FP32 hierarchy in the mixed path, its input and output
    converted).  The Krylov vectors, the operator (``glide_vjp``) and the
    residual it reports are in the state's precision, so the mixed path's
    multiplier solves the FP64 system.  With the physics'
    ``adjoint_exact_jacobian`` the operator includes the grounding-line
    derivatives (the transpose of the exact Jacobian) while the
    preconditioner keeps the solver's own Jacobian.  No counterpart in the
    reference, which runs two adjoint V-cycles (glide/physics.py:211-242)."""

    def __init__(self, physics, m=30):
        self.ph = physics
        self.lib = N.load()
        g = physics.grid
        self.mixed = physics.grid32 is not None
        self.gc = physics.grid32 if self.mixed else g   # level 0 of the cycle hierarchy
        self.n = g.nb * g.n_total
        self.m = int(m)
        dev, dt = g.device, g.dtype
        self.code = g.code
        self.V = torch.zeros(self.m + 1, self.n, dtype=dt, device=dev)
        self.Z = torch.zeros(self.m, self.n, dtype=dt, device=dev)
        self.w = torch.zeros(self.n, dtype=dt, device=dev)
        self.zero = torch.zeros(self.n, dtype=dt, device=dev)
        self.f = torch.zeros(self.n, dtype=dt, device=dev)
        self.lam = torch.zeros(self.n, dtype=dt, device=dev)
        self.r = torch.zeros(self.n, dtype=dt, device=dev)
        self.pin = torch.zeros(self.n, dtype=dt, device=dev)
        self.pout = torch.zeros(self.n, dtype=dt, device=dev)
        self.hb = torch.zeros(2 * self.m + 4, dtype=torch.float64, device=dev)
        self.y = torch.zeros(self.m, dtype=torch.float64, device=dev)
        self.parts = torch.zeros(self.lib.glide_dots_parts(self.n) * 32, dtype=torch.float64, device=dev)
        self._graphs = {}
        self._cfg = None

    def _s(self):
        return N.stream_handle()

    def _dots(self, V, k, w, out):
        N.check(self.lib.glide_dots(self.code, self.n, k, V.data_ptr(), self.n, w.data_ptr(), out.data_ptr(),
                                    self.parts.data_ptr(), self._s()), "dots")

    def _combine(self, V, k, coef, alpha, out, beta):
        N.check(self.lib.glide_combine(self.code, self.n, k, V.data_ptr(), self.n, coef.data_ptr(), float(alpha),
                                       out.data_ptr(), float(beta), self._s()), "combine")

    def _lincomb(self, out, x, a, y=None, b=0.0):
        N.check(self.lib.glide_lincomb(self.code, out.data_ptr(), x.data_ptr(), float(a),
                                       None if y is None else y.data_ptr(), float(b), self.n, self._s()), "lincomb")

    def _norm(self, x):
        self._dots(x, 1, x, self.hb[:1])
        return math.sqrt(max(float(self.hb[0].item()), 0.0))

    def _apply(self, z, out, exact, active_tol):
        """out = J_m^T z: glide_vjp gives f - z^T J_m with f = 0."""
        g = self.ph.grid
        g.compute_mask(active_tol)
        a = g.level_args()
        if self.ph.adjoint_exact_jacobian:
            a.params.gl_derivatives = 1
        zu, zv, zH = g._vec_to_fields(z)
        fu, fv, fH = g._vec_to_fields(self.zero)
        ou, ov, oH = g._vec_to_fields(out)
        N.check(self.lib.glide_vjp(C.byref(a), zu.data_ptr(), zv.data_ptr(), zH.data_ptr(), fu.data_ptr(),
                                   fv.data_ptr(), fH.data_ptr(), ou.data_ptr(), ov.data_ptr(), oH.data_ptr(),
                                   int(exact), self._s()), "adjoint operator")
        g.mask.zero_()
        self._lincomb(out, out, -1.0)

    def _precond_body(self):
        ph, gc, lib = self.ph, self.gc, self.lib
        s = self._s()
        if self.mixed:
            N.check(lib.glide_convert(N.F32, gc.f_adj.data_ptr(), self.pin.data_ptr(), self.n, 0, s), "convert")
        else:
            gc.f_adj.copy_(self.pin)
        gc.Lambda.zero_()
        N.check(lib.glide_adjoint_vcycle(ph._native, ph._nlev, 0, C.byref(self._cfg), s), "adjoint_vcycle")
        if self.mixed:
            N.check(lib.glide_convert(N.F64, self.pout.data_ptr(), gc.Lambda.data_ptr(), self.n, 1, s), "convert")
        else:
            self.pout.copy_(gc.Lambda)

    def _precond(self, key):
        """pout = one adjoint V-cycle applied to pin (from a CUDA graph)."""
        if not self.ph.use_graphs:
            self._precond_body()
            return
        entry = self._graphs.get(key)
        if entry is None:
            self._precond_body()
            torch.cuda.synchronize()
            gr = torch.cuda.CUDAGraph()
            c0 = self.lib.glide_launch_count()
            with torch.cuda.graph(gr):
                self._precond_body()
            self._graphs[key] = (gr, self.lib.glide_launch_count() - c0)
            return
        gr, nodes = entry
        gr.replay()
        self.ph.graph_launches += nodes

    def release(self):
        self._graphs.clear()

    def _linearisation_point(self):
        """The cycle hierarchy at the step's state: fl32(U) on the FP32
        hierarchy in the mixed path, the state restricted to every coarse
        level, gamma = thklim on level 0."""
        from .kernels import restrict_cell_centered, restrict_hfacet, restrict_vfacet
        ph = self.ph
        g = ph.grid
        g.gamma.fill_(ph.thklim)
        if self.mixed:
            N.check(self.lib.glide_convert(N.F32, self.gc.U.data_ptr(), g.U.data_ptr(), self.n, 0, self._s()),
                    "convert")
            self.gc.gamma.fill_(ph.thklim)
        hier = ph.grids32 if self.mixed else ph.grids
        for par, ch in zip(hier[:-1], hier[1:]):
            restrict_vfacet(par.u, u_coarse=ch.u)
            restrict_hfacet(par.v, v_coarse=ch.v)
            restrict_cell_centered(par.H, f_coarse=ch.H)

    def solve(self, cfg, tol, max_its=300, exact=False, active_tol=0.1):
        """lam for the current f_adj of the state grid, until |f - J_m^T lam|
        <= tol |f| or ``max_its`` iterations; lam is left in the state grid's
        Lambda.  Returns (iterations, relative residual reached)."""
        ph, m = self.ph, self.m
        g = ph.grid
        self._cfg = cfg
        key = (float(g.dt), int(cfg.exact_adjoint), float(cfg.adj_active_tol))
        self._linearisation_point()
        self.f.copy_(g.f_adj)
        self.lam.zero_()
        f0 = self._norm(self.f)
        if not (f0 > 0.0 and math.isfinite(f0)):
            g.Lambda.zero_()
            return 0, (0.0 if f0 == 0.0 else float("nan"))
        self.r.copy_(self.f)
        rel = 1.0
        total = 0
        hb = self.hb
        while rel > tol and total < max_its:
            beta = self._norm(self.r)
            self._lincomb(self.V[0], self.r, 1.0 / beta)
            Hm = np.zeros((m + 1, m))
            its, y = 0, None
            for j in range(m):
                self.pin.copy_(self.V[j])
                self._precond(key)
                self.Z[j].copy_(self.pout)
                self._apply(self.Z[j], self.w, exact, active_tol)
                k = j + 1
                h1, h2, hn = hb[:k], hb[m + 1:m + 1 + k], hb[2 * m + 2:2 * m + 3]
                self._dots(self.V, k, self.w, h1)
                self._combine(self.V, k, h1, -1.0, self.w, 1.0)
                self._dots(self.V, k, self.w, h2)          # second pass (CGS2)
                self._combine(self.V, k, h2, -1.0, self.w, 1.0)
                self._dots(self.w, 1, self.w, hn)
                h = hb.cpu().numpy()
                Hm[:k, j] = h[:k] + h[m + 1:m + 1 + k]
                hnorm = math.sqrt(max(h[2 * m + 2], 0.0))
                Hm[k, j] = hnorm
                its = k
                e1 = np.zeros(k + 1)
                e1[0] = beta
                y, *_ = np.linalg.lstsq(Hm[:k + 1, :k], e1, rcond=None)
                est = float(np.linalg.norm(e1 - Hm[:k + 1, :k] @ y)) / f0
                if not (np.isfinite(est) and np.all(np.isfinite(y))):
                    its = 0
                    break
                if est <= 0.5 * tol or hnorm <= 1e-30 * beta or total + its >= max_its:
                    break
                if j + 1 < m:
                    self._lincomb(self.V[j + 1], self.w, 1.0 / hnorm)
            if its == 0:
                rel = float("nan")
                break
            total += its
            self.y[:its].copy_(torch.as_tensor(y, dtype=torch.float64))
            self._combine(self.Z, its, self.y, 1.0, self.lam, 1.0)
            # true residual of the restart
            self._apply(self.lam, self.w, exact, active_tol)
            self._lincomb(self.r, self.f, 1.0, self.w, -1.0)
            new = self._norm(self.r) / f0
            if not math.isfinite(new):
                rel = new
                break
            stalled = new > 0.9 * rel
            rel = new
            if stalled:
                break
        g.Lambda.copy_(self.lam)
        g.f_adj.copy_(self.f)
        return total, rel
