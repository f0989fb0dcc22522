"""IcePhysics: the drop-in API of the SSA forward/adjoint hot path.

Same constructor and methods as glide/physics.py:49-259
(``set_geometry``, ``set_parameters``, ``forward``, ``adjoint``,
``reset_solution``, ``get_surface``, ``get_velocities_cell_centered``) and the
same loss helpers (glide/physics.py:262-411).  Arrays are accepted as NumPy
arrays, torch tensors or anything ``numpy.asarray`` understands; results are
torch CUDA tensors that are views into the persistent state (overwritten by
the next call, as in the reference).

Additions (keyword-only):
  precision  "fp32" (the reference's arithmetic, default), "fp64", or
             "mixed": FP64 state and fine-grid residual/norms with FP32
             V-cycles as the correction solver (defect correction).
  forward(tol=..., max_vcycles=...)  stop on |r|/|r0| <= tol, where |r|
             combines r_u, r_v and FB(r_H, H-gamma) (glide/physics.py:176-198)
             and r0 is the residual of the step's starting state.
  forward(guess=(u, v))  start from a supplied velocity guess; the plain
             cycle finishes the solve and the guess is dropped when the first
             cycle fails to cut the residual by ``guess_min_reduction``.
  forward(tol=..., finish=True)  once a V-cycle cuts |r| by less than
             ``stall_factor`` (the coarse-grid correction then stops helping:
             it re-injects an error near 1e-5 relative on these problems),
             continue with blocks of ``finish_block`` FP64 fine-level Vanka
             sweeps until the tolerance is met.
  settings   solver settings (``SolverSettings``); defaults = reference.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import _native as N
from .grid import Grid
from .solver import REFERENCE, SolverSettings, native_levels, restrict_parameters_to_hierarchy

RHO_ICE = 917.0
G = 9.81

_PRECISIONS = {"fp32": torch.float32, "fp64": torch.float64, "mixed": torch.float64}


def _as_tensor(x, dtype, device, shape=None):
    if isinstance(x, torch.Tensor):
        t = x.detach().to(device=device, dtype=dtype)
    else:
        t = torch.as_tensor(np.asarray(x), dtype=dtype, device=device)
    if shape is not None and t.dim() > 0 and tuple(t.shape) != tuple(shape):
        raise ValueError(f"expected shape {tuple(shape)}, got {tuple(t.shape)}")
    return t


class _NativeProducts:
    """The two vector products of the Anderson step on the library's kernels:
    dot products of stored rows with one vector (FP64 accumulation, fixed
    order) and a linear combination of stored rows."""

    def __init__(self, n, dtype, device):
        self.lib = N.load()
        self.n, self.code = int(n), N.dtype_code(dtype)
        self.parts = torch.zeros(self.lib.glide_dots_parts(self.n) * 32, dtype=torch.float64, device=device)
        self.out = torch.zeros(32, dtype=torch.float64, device=device)
        self.coef = torch.zeros(32, dtype=torch.float64, device=device)

    def dots(self, rows, w):
        k = rows.shape[0]
        N.check(self.lib.glide_dots(self.code, self.n, k, rows.data_ptr(), self.n, w.data_ptr(), self.out.data_ptr(),
                                    self.parts.data_ptr(), N.stream_handle()), "dots")
        return self.out[:k].cpu().numpy()

    def combine(self, rows, coef, out):
        k = rows.shape[0]
        self.coef[:k].copy_(torch.as_tensor(coef, dtype=torch.float64))
        N.check(self.lib.glide_combine(self.code, self.n, k, rows.data_ptr(), self.n, self.coef.data_ptr(), 1.0,
                                       out.data_ptr(), 0.0, N.stream_handle()), "combine")


class _Anderson:
    """Anderson acceleration (depth m) of the velocity over finishing blocks.

    With f_k = G_k - x_k (G_k the state after block k, x_k before it) and
    dF, dG the differences of consecutive f and G, the next state is
    G_k - dG gam, gam = argmin |f_k - dF gam| (normal equations, Tikhonov
    1e-12 trace).  The last m + 1 pairs live in preallocated ring buffers; each
    block adds one multi-dot pass for the new f's dot products (the small Gram
    matrix is kept on the host) and one linear combination, so no history is
    stacked or copied.  ``products`` supplies those two device products
    (default: the library's kernels).
    """

    def __init__(self, m, n, dtype, device, products=None):
        self.m = int(m)
        self.F = torch.zeros(self.m + 1, n, dtype=dtype, device=device)
        self.G = torch.zeros(self.m + 1, n, dtype=dtype, device=device)
        self.gram = np.zeros((self.m + 1, self.m + 1))
        self.order = []
        self.products = products if products is not None else _NativeProducts(n, dtype, device)

    def reset(self):
        self.order = []
        self.F.zero_()
        self.G.zero_()

    def step(self, x_before, x):
        """x (a view of the state) holds the block's result; replace it by the extrapolation."""
        slot = self.order.pop(0) if len(self.order) == self.m + 1 else len(self.order)
        if slot in self.order:
            self.order.remove(slot)
        self.order.append(slot)
        torch.sub(x, x_before, out=self.F[slot])
        self.G[slot].copy_(x)
        dots = self.products.dots(self.F, self.F[slot])
        self.gram[slot, :] = dots
        self.gram[:, slot] = dots
        k = len(self.order)
        if k < 2:
            return
        gf = self.gram[np.ix_(self.order, self.order)]
        D = np.zeros((k, k - 1))
        for i in range(k - 1):
            D[i, i], D[i + 1, i] = -1.0, 1.0
        Gm = D.T @ gf @ D
        tr = np.trace(Gm)
        if not (np.isfinite(tr) and tr > 0):
            return
        Gm = Gm + 1e-12 * tr * np.eye(k - 1)
        try:
            gam = np.linalg.solve(Gm, D.T @ gf[:, -1])
        except np.linalg.LinAlgError:
            return
        c = -(D @ gam)
        c[-1] += 1.0
        full = np.zeros(self.m + 1)
        full[self.order] = c
        self.products.combine(self.G, full, x)


class IcePhysics:
    """GPU shallow-shelf ice-flow model (forward step + adjoint) on one B200."""

    def __init__(self, ny, nx, dx, n_levels=5, n=3.0, eps_reg=1e-5, thklim=0.1, water_drag=1e-3, calving_rate=1.0,
                 gl_sigmoid_c=0.1, gl_derivatives=False, *, precision="fp32", device=None,
                 settings: SolverSettings | None = None, batch=1, use_graphs=True, guess_min_reduction=10.0,
                 stall_factor=0.5, finish_block=20, finish_anderson=0, finish_fp32=False, finish_newton=None,
                 finish_step=None, finish_linear=False, finish_patience=3,
                 finish_fas_until=math.inf, finish_fas_patience=10, newton=False, newton_start=1e-3,
                 newton_max_steps=8, newton_rtol=1e-2, newton_krylov=20, newton_min_gain=1.0,
                 newton_local=0, newton_after=0, newton_tries=6, adjoint_krylov=30, adjoint_max_its=300,
                 adjoint_exact_jacobian=False, branch_hops=2):
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        if not torch.cuda.is_available():
            raise N.NativeError("IcePhysics needs a CUDA device")
        if ny % (2 ** (n_levels - 1)) or nx % (2 ** (n_levels - 1)):
            raise ValueError("ny and nx must be divisible by 2**(n_levels-1)")
        self.ny, self.nx, self.dx, self.n_levels = int(ny), int(nx), float(dx), int(n_levels)
        self.n, self.eps_reg, self.thklim = float(n), float(eps_reg), float(thklim)
        self.water_drag, self.calving_rate = float(water_drag), float(calving_rate)
        self.gl_sigmoid_c, self.gl_derivatives = float(gl_sigmoid_c), bool(gl_derivatives)
        self.precision = precision
        self.settings = settings or SolverSettings()
        self.batch = int(batch)
        self.use_graphs = bool(use_graphs)
        self.guess_min_reduction = float(guess_min_reduction)
        self.stall_factor = float(stall_factor)
        self.finish_block = int(finish_block)
        self.finish_anderson = int(finish_anderson)
        self.finish_fp32 = bool(finish_fp32)
        self.finish_newton = None if finish_newton is None else int(finish_newton)
        self.finish_step = None if finish_step is None else float(finish_step)
        if finish_linear not in (False, True, "after"):
            raise ValueError('finish_linear must be False, True or "after"')
        self.finish_linear = finish_linear
        self.finish_patience = int(finish_patience)
        self.finish_fas_until = float(finish_fas_until)
        self.finish_fas_patience = int(finish_fas_patience)
        if newton and precision == "fp32":
            raise ValueError('newton=True needs an FP64 state: precision="mixed" or "fp64"')
        self.newton = bool(newton)
        self.newton_start = float(newton_start)
        self.newton_max_steps = int(newton_max_steps)
        self.newton_rtol = float(newton_rtol)
        self.newton_krylov = int(newton_krylov)
        self.newton_min_gain = float(newton_min_gain)
        self.newton_local = int(newton_local)
        self.newton_after = int(newton_after)
        self.newton_tries = int(newton_tries)
        self._nk = None
        self.adjoint_krylov = int(adjoint_krylov)
        self.adjoint_max_its = int(adjoint_max_its)
        if adjoint_exact_jacobian and self.adjoint_krylov <= 0:
            raise ValueError("adjoint_exact_jacobian needs the Krylov adjoint (adjoint_krylov > 0)")
        # the tolerance adjoint's operator with the grounding-line derivatives (the forward solve and the
        # adjoint cycles keep gl_derivatives)
        self.adjoint_exact_jacobian = bool(adjoint_exact_jacobian)
        self.branch_hops = int(branch_hops)
        self._ak = None
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.kernels = N.load()
        self.dtype = _PRECISIONS[precision]
        self._init_hierarchy()
        self._graphs = {}
        self.graph_launches = 0
        self.last_history = []
        self.last_info = {}

    # ------------------------------------------------------------------ setup
    def _make(self, dtype):
        g = Grid(self.ny, self.nx, self.dx, dt=1.0, n=self.n, eps_reg=self.eps_reg, water_drag=self.water_drag,
                 calving_rate=self.calving_rate, gl_sigmoid_c=self.gl_sigmoid_c, gl_derivatives=self.gl_derivatives,
                 dtype=dtype, device=self.device, nb=self.batch)
        gs = [g]
        return g, gs

    def _init_hierarchy(self):
        if self.precision == "mixed":
            self.grid, _ = self._make(torch.float64)
            self.grids = [self.grid]
            self.grid32, gs32 = self._make(torch.float32)
            for _ in range(self.n_levels - 1):
                gs32.append(gs32[-1].spawn_child())
            self.grids32 = gs32
            self._solve_grids = gs32
        else:
            self.grid, gs = self._make(self.dtype)
            for _ in range(self.n_levels - 1):
                gs.append(gs[-1].spawn_child())
            self.grids = gs
            self.grid32 = None
            self._solve_grids = gs
        self._native, self._nlev = native_levels(self._solve_grids[0])

    def _shape(self):
        return (self.ny, self.nx) if self.batch == 1 else (self.batch, self.ny, self.nx)

    def _all_levels(self):
        return self.grids + (self.grids32 if self.grid32 is not None else [])

    def _propagate_geometry_to_hierarchy(self):
        from .kernels import restrict_cell_centered
        for hier in ([self.grids] if self.grid32 is None else [self.grids32]):
            for par, ch in zip(hier[:-1], hier[1:]):
                restrict_cell_centered(par.bed, None, f_coarse=ch.bed)
                restrict_cell_centered(par.H, None, f_coarse=ch.H)
                restrict_cell_centered(par.H_prev, None, f_coarse=ch.H_prev)
                ch.gamma.fill_(self.thklim)

    def set_geometry(self, bed, thickness):
        """Bed and ice thickness (glide/physics.py:82-99)."""
        g = self.grid
        g.bed.copy_(_as_tensor(bed, g.dtype, self.device, self._shape()))
        g.H.copy_(_as_tensor(thickness, g.dtype, self.device, self._shape()))
        g.H_prev.copy_(g.H)
        g.gamma.fill_(self.thklim)
        if self.grid32 is not None:
            g32 = self.grid32
            g32.bed.copy_(g.bed)
            g32.H.copy_(g.H)
            g32.H_prev.copy_(g.H_prev)
            g32.gamma.fill_(self.thklim)
        self._propagate_geometry_to_hierarchy()

    def set_parameters(self, B=None, beta=None, smb=None):
        """Rate factor, basal friction, surface mass balance (glide/physics.py:101-129)."""
        g = self.grid
        if B is not None:
            Bt = _as_tensor(B, g.dtype, self.device)
            if Bt.dim() == 0:
                g.B.fill_(float(Bt))
            else:
                g.B.copy_(Bt.reshape(self._shape()))
        if beta is not None:
            g.beta.copy_(_as_tensor(beta, g.dtype, self.device, self._shape()))
        if smb is not None:
            g.smb.copy_(_as_tensor(smb, g.dtype, self.device, self._shape()))
        if self.grid32 is not None:
            for name in ("B", "beta", "smb", "bed", "H_prev"):
                getattr(self.grid32, name).copy_(getattr(g, name))
            restrict_parameters_to_hierarchy(self.grid32)
        else:
            restrict_parameters_to_hierarchy(self.grid)

    # ------------------------------------------------------------------ cycles
    def _set_dt(self, dt):
        for g in self._all_levels():
            g.dt = float(dt)
        # dt is passed to the kernels by value: rebuild the level descriptors
        self._native, self._nlev = native_levels(self._solve_grids[0])

    def _cfg(self):
        return self.settings.native(self.thklim)

    def _vcycle_native(self):
        cfg = self._cfg()
        N.check(self.kernels.glide_fascd_vcycle(self._native, self._nlev, 0, 1, C.byref(cfg), N.stream_handle()),
                "fascd_vcycle")

    def _dc_step(self):
        """Mixed precision: one FP32 FASCD cycle as the correction solver of the
        FP64 problem.  r64 = F64(U64) - f64; f32 = F32(U32) - r64 with
        U32 = fl32(U64); after the cycle U64 += fl64(U32 - w32)."""
        g64, g32 = self.grid, self.grid32
        lib = self.kernels
        s = N.stream_handle()
        g64.compute_residual()
        n = g64.nb * g64.n_total
        N.check(lib.glide_convert(N.F32, g32.U.data_ptr(), g64.U.data_ptr(), n, 0, s), "convert")
        N.check(lib.glide_convert(N.F32, g32.r.data_ptr(), g64.r.data_ptr(), n, 0, s), "convert")
        a = g32.level_args()
        N.check(lib.glide_residual(C.byref(a), g32.r_u.data_ptr(), g32.r_v.data_ptr(), g32.r_H.data_ptr(),
                                   g32.f_u.data_ptr(), g32.f_v.data_ptr(), g32.f_H.data_ptr(), s), "residual32")
        self._vcycle_native()   # sets w32 = U32 first
        N.check(lib.glide_lincomb(N.F32, g32.z.data_ptr(), g32.U.data_ptr(), 1.0, g32.w.data_ptr(), -1.0, n, s),
                "lincomb")
        N.check(lib.glide_convert(N.F64, g64.U.data_ptr(), g32.z.data_ptr(), n, 1, s), "convert")

    def _cycle(self):
        if self.precision == "mixed":
            self._dc_step()
        else:
            self._vcycle_native()

    def _run_cycle(self):
        """One V-cycle (or defect-correction step), replayed from a CUDA graph.

        ``graph_launches`` accumulates the kernel launches executed by graph
        replays (the library's own counter sees a captured launch once, at
        capture)."""
        if not self.use_graphs:
            self._cycle()
            return
        key = (float(self.grid.dt),)
        entry = self._graphs.get(key)
        if entry is None:
            self._cycle()  # warm-up launch (also checks arguments); does this cycle's work
            torch.cuda.synchronize()
            gr = torch.cuda.CUDAGraph()
            c0 = self.kernels.glide_launch_count()
            with torch.cuda.graph(gr):
                self._cycle()  # recorded, not executed
            self._graphs[key] = (gr, self.kernels.glide_launch_count() - c0)
            return
        gr, nodes = entry
        gr.replay()
        self.graph_launches += nodes

    def residual_norm(self):
        """|r| of the finest level with gamma = thklim (glide/physics.py:176-186); FP64, host float."""
        g = self.grid
        g.compute_residual()
        sq = g.residual_norms()
        return math.sqrt(float(sq.sum().item()))

    # ------------------------------------------------------------------ API
    def forward(self, dt, n_vcycles=3, verbose=False, update_geometry=True, *, tol=None, max_vcycles=100,
                guess=None, history=None, finish=True, max_finish_sweeps=4000, r0=None):
        """One implicit time step (glide/physics.py:141-209).

        Without ``tol`` runs ``n_vcycles`` cycles like the reference.  With
        ``tol`` runs cycles until |r|/|r0| <= tol; with ``finish`` a stalled
        cycle hands over to FP64 fine-level relaxation (see the module doc).
        ``r0`` (with ``tol``) continues an earlier solve of the same step from
        the current state: |r0| is then the given norm of the step's starting
        residual instead of the residual of the current state.
        ``last_info`` records cycles, finishing sweeps, the residual reached
        and whether a guess was used or dropped.
        """
        self._set_dt(dt)
        g = self.grid
        g.f_H.copy_(g.H_prev / g.dt + g.smb)
        if self.grid32 is not None:
            self.grid32.f_H.copy_(g.f_H)  # overwritten by the correction RHS, kept for API reads
        track = tol is not None or verbose or history is not None or guess is not None
        if r0 is None or tol is None:
            r0 = self.residual_norm() if track else None
        hist = [1.0] if track else []
        info = {"vcycles": 0, "finish_sweeps": 0, "guess_used": False, "fallback": False}
        if verbose:
            print(f"  Initial: |r| = {r0:.2e}")
        if guess is not None:
            saved = g.U.clone()
            gu, gv = guess
            g.u.copy_(_as_tensor(gu, g.dtype, self.device))
            g.v.copy_(_as_tensor(gv, g.dtype, self.device))
            info["guess_used"] = True
        n_max = max_vcycles if tol is not None else n_vcycles
        k = 0
        prev = 1.0
        rel = 1.0
        if tol is not None and n_max <= 0:
            # no cycles (max_vcycles=0): the finish alone, from the current state
            rel = self.residual_norm() / r0 if r0 > 0 else 0.0
            prev = rel
        stalled = False
        good = self._good_state() if tol is not None else None
        while k < n_max:
            if good is not None:
                good.copy_(g.U)
            self._run_cycle()
            k += 1
            if not track:
                continue
            rel = self.residual_norm() / r0 if r0 > 0 else 0.0
            if good is not None and (not math.isfinite(rel) or rel > 100.0 * prev) and not (
                    guess is not None and k == 1 and info["guess_used"]):
                # a diverging cycle: keep the state before it and finish by relaxation
                g.U.copy_(good)
                info["cycle_restored"] = True
                rel = prev
                stalled = True
                break
            if guess is not None and k == 1 and info["guess_used"]:
                # judge the guess by the first cycle: it must cut |r| by guess_min_reduction
                if not (rel * self.guess_min_reduction <= 1.0) or not math.isfinite(rel):
                    g.U.copy_(saved)
                    info["fallback"] = True
                    info["guess_used"] = False
                    hist.append(float("nan"))
                    rel = 1.0
                    continue
            hist.append(rel)
            if verbose:
                print(f"  V-cycle {k - 1}: |r|/|r0| = {rel:.2e}")
            if tol is not None and rel <= tol:
                break
            if tol is not None and finish and rel > self.stall_factor * prev:
                stalled = True
                break
            if tol is not None and finish and self.newton and self.newton_after == 0 and rel <= self.newton_start:
                stalled = True   # close enough for the Newton-Krylov finish
                break
            prev = rel
        if tol is not None and finish and rel > tol and (stalled or k >= n_max):
            rel = self._finish(r0, tol, max_finish_sweeps, hist, info, verbose, rel)
        if tol is not None and guess is not None and info["guess_used"] and not rel <= tol:
            # the guess led somewhere the solver cannot finish from: solve again from the plain start
            g.U.copy_(saved)
            self.forward(dt, n_vcycles, verbose, update_geometry=False, tol=tol, max_vcycles=max_vcycles,
                         guess=None, history=hist, finish=finish, max_finish_sweeps=max_finish_sweeps)
            sub = self.last_info
            k += sub["vcycles"]
            info["finish_sweeps"] = info.get("finish_sweeps", 0) + sub["finish_sweeps"]
            info.update(fallback=True, guess_used=False, late_fallback=True)
            rel = sub["rel_residual"]
        info["vcycles"] = k
        info["rel_residual"] = rel if track else None
        self.last_history = hist
        self.last_info = info
        if history is not None:
            history.extend(hist)
        if update_geometry:
            g.H_prev.copy_(g.H)
            if self.grid32 is not None:
                self.grid32.H_prev.copy_(g.H)
        return g.u, g.v, g.H

    def _finish(self, r0, tol, max_sweeps, hist, info, verbose, rel):
        """Fine-level Vanka relaxation in blocks until |r|/|r0| <= tol, from
        the current state, whose relative residual is ``rel``.

        Mixed precision with ``finish_fp32``: blocks of FP32 sweeps on the
        correction problem f32 = F32(fl32(U64)) - r64 while they still cut the
        FP64 residual, then FP64 sweeps.  ``finish_anderson`` = m > 0 applies
        Anderson acceleration (depth m) over the blocks to the velocity part.
        ``finish_linear``: True -- the FP32 blocks solve the linearised
        correction problem instead (``_linear_block``) and hand over to FP64
        after ``finish_patience`` blocks without a new best; "after" -- FAS-form
        FP32 blocks first, the linearised ones from the FAS form's floor on.
        A FAS-form block that gains less than 1/0.7 counts as the floor only
        at |r|/|r0| <= ``finish_fas_until``: above it the gain is small because
        the smoother is slow, far from the solution, where the linearised
        correction can diverge (the default, inf, always counts a small gain).
        The FAS form also ends after ``finish_fas_patience`` blocks without a
        new best.  For the 1024^2 benchmark geometries, whose FP32 floor lies
        near 1e-4, 2e-4 and 8 blocks suit both fresh and warm-started steps.
        Ten blocks without
        progress restore the best state and continue in FP64 with the
        reference's damped local Newton and no extrapolation.  Divergence or
        stagnation in that safe mode restores the best state again, halves the
        sweeps' omega and lets the Newton-Krylov finish try again (up to
        ``newton_tries`` attempts in all).  When omega would fall below 1/16
        of the setting, the cell with the largest residual is moved to the
        other root of its mass balance (``_branch_hop``, at most
        ``branch_hops`` times) and the finish starts over from there; the
        best state over all attempts is kept.  It ends at ``max_sweeps``.
        """
        g = self.grid
        st = self.settings
        g.gamma.fill_(self.thklim)
        done = 0
        use32 = self.grid32 is not None and self.finish_fp32
        # FP32 block form: "fas" (correction problem in FAS form), "linear" (linearised correction)
        form32 = "linear" if self.finish_linear is True else "fas"
        m = self.finish_anderson
        nU = g.nb * (g.nu + g.nv)
        aa = _Anderson(m, nU, g.dtype, g.device) if m > 0 else None
        x0 = torch.empty(nU, dtype=g.dtype, device=g.device) if m > 0 else None
        prev = rel
        best, good = rel, self._good_state()
        good.copy_(g.U)
        since_best = 0
        local = self._finish_local()
        blocks = {"fp32": 0, "fp64": 0}
        info["finish_blocks"] = blocks
        fas_until = self.finish_fas_until
        nk_last = math.inf   # |r|/|r0| at the last Newton-Krylov attempt
        nk_tries = 0
        damp = 1.0           # omega factor of the safe mode's FP64 sweeps
        hops = 0
        hop_keep, hop_rel = None, math.inf   # best state before the last branch hop

        def hop():
            """Move the worst cell to its other mass-balance root; restart the finish state."""
            nonlocal hops, hop_keep, hop_rel, rel, best, since_best, nk_last, nk_tries, damp, local, use32, m
            nonlocal prev, form32
            if hops >= self.branch_hops:
                return False
            if best < hop_rel:
                if hop_keep is None:
                    hop_keep = torch.empty_like(g.U)
                hop_keep.copy_(good)
                hop_rel = best
            g.U.copy_(good)
            if not self._branch_hop():
                return False
            hops += 1
            info["branch_hops"] = hops
            rel = self.residual_norm() / r0 if r0 > 0 else 0.0
            best = prev = rel
            good.copy_(g.U)
            since_best, nk_last, nk_tries, damp = 0, math.inf, 0, 1.0
            local = self._finish_local()
            use32 = self.grid32 is not None and self.finish_fp32
            form32 = "linear" if self.finish_linear is True else "fas"
            m = self.finish_anderson
            if aa is not None:
                aa.reset()
            hist.append(rel)
            return True
        while done < max_sweeps and rel > tol:
            if (self.newton and rel <= self.newton_start and rel < 0.5 * nk_last and
                    nk_tries < self.newton_tries and done >= self.newton_after):
                # Newton-Krylov from here; a failed attempt falls back to the blocks below, and a
                # new attempt follows once they have halved the residual
                nk_tries += 1
                rel = self._newton_krylov().solve(r0, tol, rel, hist, info, max_steps=self.newton_max_steps,
                                                  rtol=self.newton_rtol, min_gain=self.newton_min_gain,
                                                  local_rounds=self.newton_local)
                nk_last = rel
                if rel < best:
                    best = rel
                    good.copy_(g.U)
                    since_best = 0
                if aa is not None:
                    aa.reset()
                prev = rel
                continue
            if m > 0:
                x0.copy_(g.U[:nU])
            blocks["fp32" if use32 else "fp64"] += 1
            if use32 and form32 == "linear":
                blocks["linear"] = blocks.get("linear", 0) + 1
                self._linear_block(self.finish_block)
            elif use32:
                self._fp32_sweeps(self.finish_block, local)
            else:
                g.vanka_sweep(self.finish_block, omega=st.omega * damp, shift=st.shift, **local)
            done += self.finish_block
            if m > 0:
                # an extrapolation that raises |r| is kept on purpose: measured, it shortens the finish
                # (the residual norm understates the smooth error it removes)
                aa.step(x0, g.U[:nU])
            rel = self.residual_norm() / r0 if r0 > 0 else 0.0
            hist.append(rel)
            if verbose:
                print(f"  finish {done} sweeps ({'fp32' if use32 else 'fp64'}): |r|/|r0| = {rel:.2e}")
            if not math.isfinite(rel) or rel > 100.0 * best:
                # diverging relaxation: back to the best state, then the reference's damped local Newton
                # without extrapolation
                g.U.copy_(good)
                rel = best
                safe = dict(n_inner=REFERENCE.n_newton, step=REFERENCE.newton_step)
                if local == safe and m == 0:
                    # diverged in the safe mode too: on in FP64, then with more damping; Newton-Krylov
                    # may try again from the best state
                    if use32:
                        use32 = False
                    else:
                        damp *= 0.5
                        if damp < 1.0 / 16:
                            if hop():
                                continue
                            break
                        info["finish_damp"] = damp
                    nk_last = math.inf
                    since_best = 0
                    continue
                local, m = safe, 0
                info["finish_safe"] = True
                continue
            if rel < best:
                if rel < 0.99 * best:
                    since_best = 0
                best = rel
                good.copy_(g.U)
            since_best += 1
            if since_best > 10:
                # no progress over 10 blocks: back to the best state and on in FP64 with the reference's
                # damped local Newton and no extrapolation; a stagnation in that mode halves omega (and
                # lets Newton-Krylov try again) until omega would fall below 1/16 (then a late guess
                # fallback may follow)
                safe = dict(n_inner=REFERENCE.n_newton, step=REFERENCE.newton_step)
                if local == safe and not use32 and m == 0:
                    damp *= 0.5
                    if damp < 1.0 / 16:
                        if hop():
                            continue
                        info["finish_stagnated"] = True
                        break
                    info["finish_damp"] = damp
                    nk_last = math.inf
                g.U.copy_(good)
                rel = best
                local, use32, m = safe, False, 0
                since_best = 0
                info["finish_safe"] = True
                continue
            # the FAS-form FP32 correction floors near eps32 x |operator terms|: once a block gains little
            # (at |r|/|r0| <= fas_until; above it a small gain means slow smoothing) or none of the last
            # finish_fas_patience blocks set a new best,
            # hand over to FP64 -- or, with finish_linear="after", to the linearised FP32 correction, which
            # has no such floor and is accurate this close to the solution; the linear form hands over to
            # FP64 when it has not set a new best for finish_patience blocks (Anderson steps may raise |r|)
            if use32 and form32 == "fas" and ((rel > 0.7 * prev and rel <= fas_until) or
                                              since_best >= self.finish_fas_patience):
                if self.finish_linear == "after":
                    form32 = "linear"
                    since_best = 0
                else:
                    use32 = False
                if aa is not None:
                    aa.reset()
            elif use32 and form32 == "linear" and since_best >= self.finish_patience:
                use32 = False
                if aa is not None:
                    aa.reset()
            prev = rel
        if hop_keep is not None and not rel <= hop_rel:
            g.U.copy_(hop_keep)   # the hops did not pay: back to the best state before them
            rel = hop_rel
        info["finish_sweeps"] = done
        return rel

    def _branch_hop(self):
        """Move the cell with the largest residual to the other root of its
        own mass balance, velocities and the neighbours' fluxes held fixed.

        With the net outflow D of the cell at the current state,
        r_H(H) = H/dt + c (1 - g(H)) H + D - f_H (glide/cuda/flux.cu:187-211)
        has a grounded root H = (f_H - D) dt and a floating root
        H = (f_H - D) / (1/dt + c) when the flotation thickness -bed/0.917
        lies between them.  A finish that stalls at a handful of cells at the
        grounding line sits where the branch it follows ends (the two roots
        merge); the step's solution there is on the other branch.  Returns
        False when the cell has no other root."""
        g = self.grid
        g.gamma.fill_(self.thklim)
        g.compute_residual()
        Hm = g.H - g.gamma
        rH = g.r_H
        fb = (Hm + rH - torch.sqrt(Hm * Hm + rH * rH)).abs().flatten()
        k = int(torch.argmax(fb).item())
        H_new = other_mass_root(float(g.H.flatten()[k]), float(g.bed.flatten()[k]), float(g.f_H.flatten()[k]),
                                float(rH.flatten()[k]), float(g.dt), self.calving_rate, self.gl_sigmoid_c,
                                self.thklim)
        if H_new is None:
            return False
        g.H.view(-1)[k] = H_new
        return True

    def _newton_krylov(self):
        from .newton import NewtonKrylov
        if self._nk is None:
            self._nk = NewtonKrylov(self, m=self.newton_krylov)
        return self._nk

    def _finish_local(self):
        """Local Newton iterations and step fraction of the finishing sweeps
        (``finish_newton``/``finish_step``; default: the cycle's settings)."""
        st = self.settings
        return dict(n_inner=st.n_newton if self.finish_newton is None else self.finish_newton,
                    step=st.newton_step if self.finish_step is None else self.finish_step)

    def _good_state(self):
        """Preallocated copy of the state vector (the last state known to be finite)."""
        if getattr(self, "_good", None) is None or self._good.shape != self.grid.U.shape:
            self._good = torch.empty_like(self.grid.U)
        return self._good

    def _linear_block(self, n):
        """Defect correction in linear form: r64 = F64(U64) - f64; n FP32
        additive Vanka sweeps for r + J d = 0 linearised at fl32(U64) (local
        matrices factored once, r + J d from one FP32 JVP pass); U64 += fl64(d).
        Unlike the FAS-form correction its rounding error scales with d, not
        with the size of the operator's terms."""
        g64, g32 = self.grid, self.grid32
        lib = self.kernels
        s = N.stream_handle()
        st = self.settings
        ntot = g64.nb * g64.n_total
        g64.compute_residual()
        N.check(lib.glide_convert(N.F32, g32.U.data_ptr(), g64.U.data_ptr(), ntot, 0, s), "convert")
        N.check(lib.glide_convert(N.F32, g32.r.data_ptr(), g64.r.data_ptr(), ntot, 0, s), "convert")
        g32.gamma.fill_(self.thklim)
        # f32 = F32(U32) - r: the local mass residual of the factorisation equals r_H
        a = g32.level_args()
        N.check(lib.glide_residual(C.byref(a), g32.r_u.data_ptr(), g32.r_v.data_ptr(), g32.r_H.data_ptr(),
                                   g32.f_u.data_ptr(), g32.f_v.data_ptr(), g32.f_H.data_ptr(), s), "residual32")
        g32.vanka_lu(st.shift)
        g32.d_U.zero_()
        for k in range(n):
            if k == 0:
                rho = g32.r
            else:
                g32.jvp_add(g32.r, g32.z)   # rho = r + J d
                rho = g32.z
            g32.vanka_linear_sweep(rho, g32.d_U, st.omega)
        N.check(lib.glide_convert(N.F64, g64.U.data_ptr(), g32.d_U.data_ptr(), ntot, 1, s), "convert")

    def _fp32_sweeps(self, n, local=None):
        """FP32 fine-level sweeps on the FP64 problem's correction equation."""
        g64, g32 = self.grid, self.grid32
        lib = self.kernels
        s = N.stream_handle()
        st = self.settings
        ntot = g64.nb * g64.n_total
        g64.compute_residual()
        N.check(lib.glide_convert(N.F32, g32.U.data_ptr(), g64.U.data_ptr(), ntot, 0, s), "convert")
        N.check(lib.glide_convert(N.F32, g32.r.data_ptr(), g64.r.data_ptr(), ntot, 0, s), "convert")
        g32.w.copy_(g32.U)
        g32.gamma.fill_(self.thklim)
        a = g32.level_args()
        N.check(lib.glide_residual(C.byref(a), g32.r_u.data_ptr(), g32.r_v.data_ptr(), g32.r_H.data_ptr(),
                                   g32.f_u.data_ptr(), g32.f_v.data_ptr(), g32.f_H.data_ptr(), s), "residual32")
        g32.vanka_sweep(n, omega=st.omega, shift=st.shift, **(local or self._finish_local()))
        N.check(lib.glide_lincomb(N.F32, g32.z.data_ptr(), g32.U.data_ptr(), 1.0, g32.w.data_ptr(), -1.0, ntot, s),
                "lincomb")
        N.check(lib.glide_convert(N.F64, g64.U.data_ptr(), g32.z.data_ptr(), ntot, 1, s), "convert")

    def adjoint(self, dL_du, dL_dv, dL_dH, n_vcycles=2, *, tol=None, max_vcycles=100, exact=False,
                max_finish_sweeps=4000):
        """grad_beta of a loss through one implicit step (glide/physics.py:211-242).

        ``exact=True`` uses the exact transpose at clamped boundary reads in
        the VJP and the gradient (the reference drops some boundary terms).
        With ``tol`` the multiplier is solved until |f_adj - J_m^T lam| <=
        tol |f_adj| (J_m: rows of the active cells, H <= gamma +
        ``settings.adj_active_tol``, replaced by the identity, as the adjoint
        smoother sees them).  With ``adjoint_krylov`` > 0 (the default) by
        FGMRES preconditioned by one adjoint V-cycle per iteration
        (``newton.AdjointKrylov``); if that ends above ``tol``, or with
        ``adjoint_krylov=0``, by adjoint cycles from lam = 0 until a cycle
        cuts the residual by less than ``stall_factor``, then fine-level
        adjoint sweeps.  A cycle or block of sweeps whose residual is
        non-finite or grows 100x over the best one is undone (the best
        multiplier is kept): a diverging cycle hands over to the sweeps, a
        diverging block ends the solve.  ``last_adjoint_info`` records the
        work.
        """
        st = self.settings
        saved_exact = st.exact_adjoint
        st.exact_adjoint = bool(exact)
        info = {"vcycles": 0, "finish_sweeps": 0, "rel_residual": None}
        try:
            g = self.grid
            g.f_adj_u.copy_(-_as_tensor(dL_du, g.dtype, self.device))
            g.f_adj_v.copy_(-_as_tensor(dL_dv, g.dtype, self.device))
            g.f_adj_H.copy_(-_as_tensor(dL_dH, g.dtype, self.device))
            g.Lambda.zero_()
            cfg = st.native(self.thklim)
            if tol is not None and self.adjoint_krylov > 0:
                from .newton import AdjointKrylov
                if self._ak is None or self._ak.m != self.adjoint_krylov:
                    self._ak = AdjointKrylov(self, m=self.adjoint_krylov)
                its, rel = self._ak.solve(cfg, tol, max_its=self.adjoint_max_its, exact=exact,
                                          active_tol=st.adj_active_tol)
                info["krylov_its"] = its
                if math.isfinite(rel) and rel <= tol:
                    info["rel_residual"] = rel
                    self.last_adjoint_info = info
                    return g.compute_grad_beta(exact_boundary=exact, mask_tol=st.adj_active_tol)
                info["krylov_rel_residual"] = rel
                if self.adjoint_exact_jacobian:
                    # the cycles below solve the solver's own adjoint, not the exact one
                    info["rel_residual"] = rel
                    self.last_adjoint_info = info
                    return g.compute_grad_beta(exact_boundary=exact, mask_tol=st.adj_active_tol)
                g.Lambda.zero_()
            f0 = None
            n_max = max_vcycles if tol is not None else n_vcycles
            prev = 1.0
            rel = None
            # with a tolerance: the best multiplier so far; a cycle or a block of
            # sweeps whose residual is non-finite or grows 100x is undone
            best_rel, best = 1.0, None
            if tol is not None:
                if getattr(self, "_lam_best", None) is None:
                    self._lam_best = torch.empty_like(g.Lambda)
                best = self._lam_best
                best.zero_()
            for k in range(n_max):
                if self.precision == "mixed":
                    self._adjoint_dc_step(cfg)
                else:
                    N.check(self.kernels.glide_adjoint_vcycle(self._native, self._nlev, 0, C.byref(cfg),
                                                              N.stream_handle()), "adjoint_vcycle")
                info["vcycles"] = k + 1
                if tol is None:
                    continue
                rel, f0 = self._adjoint_rel(f0)
                if not math.isfinite(rel) or rel > 100.0 * best_rel:
                    g.Lambda.copy_(best)
                    rel = best_rel
                    info["cycle_restored"] = True
                    break
                if rel < best_rel:
                    best_rel = rel
                    best.copy_(g.Lambda)
                if rel <= tol or rel > self.stall_factor * prev:
                    break
                prev = rel
            if tol is not None and rel is not None and rel > tol:
                done = 0
                while done < max_finish_sweeps and rel > tol:
                    g.compute_mask(st.adj_active_tol)
                    g.vanka_sweep_adjoint(self.finish_block, omega=st.adj_omega, exact_boundary=exact)
                    g.mask.zero_()
                    done += self.finish_block
                    rel, f0 = self._adjoint_rel(f0)
                    if not math.isfinite(rel) or rel > 100.0 * best_rel:
                        g.Lambda.copy_(best)
                        rel = best_rel
                        info["finish_restored"] = True
                        break
                    if rel < best_rel:
                        best_rel = rel
                        best.copy_(g.Lambda)
                info["finish_sweeps"] = done
            info["rel_residual"] = rel
            self.last_adjoint_info = info
            return g.compute_grad_beta(exact_boundary=exact, mask_tol=st.adj_active_tol)
        finally:
            st.exact_adjoint = saved_exact

    def _adjoint_rel(self, f0):
        g = self.grid
        g.compute_mask(self.settings.adj_active_tol)
        g.compute_adjoint_residual(self.settings.exact_adjoint)
        g.mask.zero_()
        r = torch.sqrt(torch.sum(g.r_adj.double() ** 2)).item()
        if f0 is None:
            f0 = torch.sqrt(torch.sum(g.f_adj.double() ** 2)).item()
        return (r / f0 if f0 > 0 else 0.0), f0

    def _adjoint_dc_step(self, cfg):
        """Mixed precision adjoint: r64 = f_adj - J64^T lam64, FP32 adjoint
        cycle on J32^T d = fl32(r64), lam64 += fl64(d)."""
        g64, g32 = self.grid, self.grid32
        lib = self.kernels
        s = N.stream_handle()
        n = g64.nb * g64.n_total
        g64.mask.zero_()
        g64.compute_adjoint_residual(self.settings.exact_adjoint)
        N.check(lib.glide_convert(N.F32, g32.U.data_ptr(), g64.U.data_ptr(), n, 0, s), "convert")
        N.check(lib.glide_convert(N.F32, g32.f_adj.data_ptr(), g64.r_adj.data_ptr(), n, 0, s), "convert")
        g32.Lambda.zero_()
        N.check(lib.glide_adjoint_vcycle(self._native, self._nlev, 0, C.byref(cfg), s), "adjoint_vcycle")
        N.check(lib.glide_convert(N.F64, g64.Lambda.data_ptr(), g32.Lambda.data_ptr(), n, 1, s), "convert")

    def reset_solution(self):
        """glide/physics.py:244-248."""
        g = self.grid
        g.u.zero_()
        g.v.zero_()
        g.H.copy_(g.H_prev)

    def get_surface(self):
        """s = H + max(bed, -0.917 H) (glide/physics.py:250-253)."""
        g = self.grid
        return g.H + torch.maximum(g.bed, -RHO_ICE / 1000.0 * g.H)

    def get_velocities_cell_centered(self):
        """glide/physics.py:255-259."""
        g = self.grid
        return 0.5 * (g.u[..., 1:] + g.u[..., :-1]), 0.5 * (g.v[..., 1:, :] + g.v[..., :-1, :])

    def release_graphs(self):
        self._graphs.clear()
        if self._nk is not None:
            self._nk.release()
        if self._ak is not None:
            self._ak.release()


def other_mass_root(H, bed, f_H, r_H, dt, calving_rate, sig_c, thklim):
    """The other root of one cell's mass balance with its net outflow fixed.

    r_H(H) = H/dt + c (1 - g(H)) H + D - f_H (glide/cuda/flux.cu:187-211,
    g the grounding sigmoid of bed + 0.917 H); D is taken from the cell's
    residual r_H at its thickness H.  Grounded (g > 1/2): the floating root
    (f_H - D) / (1/dt + c), if it lies below the flotation thickness;
    floating: the grounded root (f_H - D) dt, if it lies above it.  None when
    that root does not exist or is not above thklim."""
    rr = RHO_ICE / 1000.0
    z = max(min(sig_c * (bed + rr * H), 20.0), -20.0)
    gnd = 1.0 / (1.0 + math.exp(-z))
    S = f_H - (r_H - H / dt - calving_rate * (1.0 - gnd) * H + f_H)   # f_H - D
    flot = -bed / rr
    if gnd > 0.5:
        H_new = S / (1.0 / dt + calving_rate)
        ok = H_new < flot
    else:
        H_new = S * dt
        ok = H_new > flot
    if not (ok and math.isfinite(H_new) and H_new > thklim):
        return None
    return H_new


# ---------------------------------------------------------------------------
# loss helpers (glide/physics.py:262-411)
# ---------------------------------------------------------------------------

def _nan0(d):
    return torch.where(torch.isnan(d), torch.zeros_like(d), d)


def huber_loss(u, v, u_obs, v_obs, eps=10.0):
    du, dv = _nan0(u - u_obs), _nan0(v - v_obs)
    return torch.sqrt(du ** 2 + eps).mean() + torch.sqrt(dv ** 2 + eps).mean()


def huber_grad(u, v, u_obs, v_obs, eps=10.0):
    du, dv = _nan0(u - u_obs), _nan0(v - v_obs)
    n = u.numel()
    return du / torch.sqrt(du ** 2 + eps) / n, dv / torch.sqrt(dv ** 2 + eps) / n


def abs_loss(u, v, u_obs, v_obs):
    du, dv = _nan0(u.double() - u_obs.double()), _nan0(v.double() - v_obs.double())
    return du.abs().mean() + dv.abs().mean()


def abs_grad(u, v, u_obs, v_obs, eps=10.0):
    du, dv = _nan0(u - u_obs), _nan0(v - v_obs)
    n = u.numel()
    return torch.sign(du) / n, torch.sign(dv) / n


def tikhonov_regularization(field):
    dx_ = field[:, 1:] - field[:, :-1]
    dy_ = field[1:, :] - field[:-1, :]
    loss = 0.5 * (torch.sum(dx_ ** 2) + torch.sum(dy_ ** 2))
    grad = torch.zeros_like(field)
    grad[:, 1:-1] -= field[:, 2:] - 2 * field[:, 1:-1] + field[:, :-2]
    grad[:, 0] -= field[:, 1] - field[:, 0]
    grad[:, -1] -= field[:, -2] - field[:, -1]
    grad[1:-1, :] -= field[2:, :] - 2 * field[1:-1, :] + field[:-2, :]
    grad[0, :] -= field[1, :] - field[0, :]
    grad[-1, :] -= field[-2, :] - field[-1, :]
    return float(loss), grad
