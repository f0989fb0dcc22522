"""One multigrid level: state vectors, parameter fields and kernel dispatch.

Mirrors ``Grid`` of the reference (glide/grid.py:14-355): the same attribute
names (``U, u, v, H, f, f_u, ..., Lambda, lambda_u, ..., mask, gamma``) are
views into monolithic device vectors ``[u | v | H]``, and the same methods
(``compute_residual``, ``compute_F``, ``compute_jvp``, ``compute_vjp``,
``vanka_sweep``, ``vanka_sweep_local``, ``vanka_sweep_adjoint``,
``compute_mask``, ``compute_grad_beta``, ``spawn_child``) dispatch to the
sm_100a kernels through the C ABI.  A level may hold a batch of ``nb``
independent problems of the same size (views then carry a leading batch
dimension).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N


class Grid:
    def __init__(self, ny, nx, dx, dt=1.0, parent=None, n=3.0, eps_reg=1e-5, water_drag=1e-3, calving_rate=1.0,
                 gl_sigmoid_c=0.1, gl_derivatives=False, dtype=torch.float32, device=None, nb=1):
        self.parent = parent
        self.child = None
        self.ny, self.nx, self.nb = int(ny), int(nx), int(nb)
        self.dx = float(dx)
        self.dt = float(dt)
        self.dtype = dtype
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self._n, self._eps_reg = float(n), float(eps_reg)
        self._water_drag, self._calving_rate = float(water_drag), float(calving_rate)
        self._gl_sigmoid_c, self._gl_derivatives = float(gl_sigmoid_c), bool(gl_derivatives)
        self.nu = ny * (nx + 1)
        self.nv = (ny + 1) * nx
        self.nU = self.nu + self.nv
        self.nh = ny * nx
        self.n_total = self.nu + self.nv + self.nh
        self._lib = N.load()
        self._allocate_arrays()

    # ------------------------------------------------------------------ memory
    def _vec(self):
        return torch.zeros(self.nb * self.n_total, dtype=self.dtype, device=self.device)

    def _cells(self):
        shape = (self.ny, self.nx) if self.nb == 1 else (self.nb, self.ny, self.nx)
        return torch.zeros(shape, dtype=self.dtype, device=self.device)

    def _vec_to_fields(self, x):
        """Field views of a monolithic vector (glide/grid.py:160-165)."""
        nb, ny, nx = self.nb, self.ny, self.nx
        u = x[:nb * self.nu]
        v = x[nb * self.nu:nb * self.nU]
        H = x[nb * self.nU:]
        if nb == 1:
            return u.view(ny, nx + 1), v.view(ny + 1, nx), H.view(ny, nx)
        return u.view(nb, ny, nx + 1), v.view(nb, ny + 1, nx), H.view(nb, ny, nx)

    def _allocate_arrays(self):
        for name, parts in (("U", ("u", "v", "H")), ("d_U", ("d_u", "d_v", "d_H")),
                            ("delta_U", ("delta_u", "delta_v", "delta_H")),
                            ("Lambda", ("lambda_u", "lambda_v", "lambda_H")),
                            ("f", ("f_u", "f_v", "f_H")), ("f_adj", ("f_adj_u", "f_adj_v", "f_adj_H")),
                            ("F", ("F_u", "F_v", "F_H")), ("Z", ("Z_u", "Z_v", "Z_H")),
                            ("r", ("r_u", "r_v", "r_H")), ("r_adj", ("r_adj_u", "r_adj_v", "r_adj_H")),
                            ("j", ("j_u", "j_v", "j_H")), ("l", ("l_u", "l_v", "l_H")),
                            ("w", ("w_u", "w_v", "w_H")), ("z", ("z_u", "z_v", "z_H"))):
            vec = self._vec()
            setattr(self, name, vec)
            for pn, view in zip(parts, self._vec_to_fields(vec)):
                setattr(self, pn, view)
        self.Lambda_out = self.Lambda  # adjoint sweeps update lambda in place
        self.lambda_u_out, self.lambda_v_out, self.lambda_H_out = self.lambda_u, self.lambda_v, self.lambda_H
        for name in ("H_prev", "chi", "phi", "bed", "beta", "B", "smb", "mask", "error_mask", "gamma"):
            setattr(self, name, self._cells())
        self._scratch = torch.zeros(5 * self.nb * self.nh, dtype=self.dtype, device=self.device)
        nflags = (self.ny // 14 + 1) * (self.nx // 14 + 1) * self.nb
        self._flags = torch.zeros(nflags, dtype=torch.int32, device=self.device)
        self._any_active = torch.zeros(self.nb, dtype=torch.int32, device=self.device)
        self._norm_out = torch.zeros(3, dtype=torch.float64, device=self.device)
        self._ls_tmp = self._ls_norms = None
        self._norm_parts = torch.zeros(3 * self._lib.glide_norm_parts(max(self.nu, self.nh) * self.nb),
                                       dtype=torch.float64, device=self.device)

    # ------------------------------------------------------------------ ABI glue
    @property
    def code(self) -> int:
        return N.dtype_code(self.dtype)

    def params(self) -> N.PhysicsParams:
        return N.PhysicsParams(self._n, self._eps_reg, self._water_drag, self._calving_rate, self._gl_sigmoid_c,
                               int(self._gl_derivatives))

    def level_args(self) -> N.LevelArgs:
        a = N.LevelArgs()
        a.ny, a.nx, a.nb, a.dtype = self.ny, self.nx, self.nb, self.code
        a.dx, a.dt = self.dx, float(self.dt)
        a.params = self.params()
        a.u, a.v, a.H = self.u.data_ptr(), self.v.data_ptr(), self.H.data_ptr()
        a.bed, a.B, a.beta = self.bed.data_ptr(), self.B.data_ptr(), self.beta.data_ptr()
        a.mask, a.gamma = self.mask.data_ptr(), self.gamma.data_ptr()
        return a

    def native_level(self) -> N.Level:
        L = N.Level()
        L.a = self.level_args()
        L.U, L.f, L.w, L.r, L.z = (t.data_ptr() for t in (self.U, self.f, self.w, self.r, self.z))
        L.chi, L.err_mask = self.chi.data_ptr(), self.error_mask.data_ptr()
        L.lam, L.f_adj, L.r_adj = self.Lambda.data_ptr(), self.f_adj.data_ptr(), self.r_adj.data_ptr()
        L.H_prev, L.smb = self.H_prev.data_ptr(), self.smb.data_ptr()
        L.scratch, L.flags, L.any_active = self._scratch.data_ptr(), self._flags.data_ptr(), self._any_active.data_ptr()
        if self.parent is None:  # coarse-correction line search on the finest level only
            if self._ls_tmp is None:
                self._ls_tmp = self._vec()
                self._ls_norms = torch.zeros(3 * N.LS_CANDIDATES + 1, dtype=torch.float64, device=self.device)
            L.ls_tmp, L.ls_norms = self._ls_tmp.data_ptr(), self._ls_norms.data_ptr()
            L.norm_parts = self._norm_parts.data_ptr()
        return L

    def newton_buffers(self):
        """Buffers of the linear multigrid of the Newton-Krylov finishing
        solver (allocated on first use): local factors, right-hand side,
        linear residual, correction, residual at the linearisation state, and
        the active set (kept apart from ``mask``, which the FAS cycle reads)."""
        if getattr(self, "_nk", None) is None:
            self._nk = {"lu": torch.zeros(25 * self.nb * self.nh, dtype=self.dtype, device=self.device),
                        "lin_rhs": self._vec(), "lin_rho": self._vec(), "lin_d": self._vec(), "r_raw": self._vec(),
                        "mask": self._cells()}
        return self._nk

    def newton_level(self, gl_sigmoid_c):
        """native_level() with the Newton-Krylov buffers attached, the active
        set in its own mask and the exact grounding-line derivatives in the
        Jacobian (they change J, not the residual)."""
        L = self.native_level()
        b = self.newton_buffers()
        L.lu, L.lin_rhs, L.lin_rho = b["lu"].data_ptr(), b["lin_rhs"].data_ptr(), b["lin_rho"].data_ptr()
        L.lin_d, L.r_raw = b["lin_d"].data_ptr(), b["r_raw"].data_ptr()
        L.a.mask = b["mask"].data_ptr()
        L.a.params.gl_derivatives = 1
        L.a.params.gl_sigmoid_c = float(gl_sigmoid_c)
        return L

    def _s(self):
        return N.stream_handle()

    # ------------------------------------------------------------------ hierarchy
    def spawn_child(self):
        """2x coarsening.  Like glide/grid.py:167-180, the child keeps n,
        eps_reg, water_drag and calving_rate but not gl_sigmoid_c /
        gl_derivatives (it falls back to 0.1 / False)."""
        child = Grid(self.ny // 2, self.nx // 2, self.dx * 2, self.dt, parent=self, n=self._n,
                     eps_reg=self._eps_reg, water_drag=self._water_drag, calving_rate=self._calving_rate,
                     dtype=self.dtype, device=self.device, nb=self.nb)
        self.child = child
        return child

    # ------------------------------------------------------------------ operators
    def compute_residual(self, return_fischer_burmeister=False):
        """r = F(U) - f (glide/grid.py:190-208)."""
        a = self.level_args()
        N.check(self._lib.glide_residual(C.byref(a), self.f_u.data_ptr(), self.f_v.data_ptr(), self.f_H.data_ptr(),
                                         self.r_u.data_ptr(), self.r_v.data_ptr(), self.r_H.data_ptr(), self._s()),
                "residual")
        if return_fischer_burmeister:
            a_, b_ = self.r_H, self.H - self.gamma
            return a_ + b_ - torch.sqrt(a_ ** 2 + b_ ** 2)

    def compute_F(self):
        """F(U) with f = 0 (glide/grid.py:210-223)."""
        a = self.level_args()
        self.Z.zero_()
        N.check(self._lib.glide_residual(C.byref(a), self.Z_u.data_ptr(), self.Z_v.data_ptr(), self.Z_H.data_ptr(),
                                         self.F_u.data_ptr(), self.F_v.data_ptr(), self.F_H.data_ptr(), self._s()),
                "compute_F")

    def compute_jvp(self):
        """j = J(U) d_U (glide/grid.py:225-238)."""
        a = self.level_args()
        N.check(self._lib.glide_jvp(C.byref(a), self.d_u.data_ptr(), self.d_v.data_ptr(), self.d_H.data_ptr(),
                                    self.j_u.data_ptr(), self.j_v.data_ptr(), self.j_H.data_ptr(), self._s()), "jvp")

    def jvp_add(self, base, out):
        """out = base + J(U) d_U in one pass (base, out: monolithic vectors like U)."""
        bu, bv, bH = self._vec_to_fields(base)
        ou, ov, oH = self._vec_to_fields(out)
        a = self.level_args()
        N.check(self._lib.glide_jvp_add(C.byref(a), self.d_u.data_ptr(), self.d_v.data_ptr(), self.d_H.data_ptr(),
                                        bu.data_ptr(), bv.data_ptr(), bH.data_ptr(), ou.data_ptr(), ov.data_ptr(),
                                        oH.data_ptr(), self._s()), "jvp_add")

    def compute_vjp(self, exact_boundary=False):
        """l = Lambda^T J(U) (glide/grid.py:240-254)."""
        a = self.level_args()
        N.check(self._lib.glide_vjp(C.byref(a), self.lambda_u.data_ptr(), self.lambda_v.data_ptr(),
                                    self.lambda_H.data_ptr(), None, None, None, self.l_u.data_ptr(),
                                    self.l_v.data_ptr(), self.l_H.data_ptr(), int(exact_boundary), self._s()), "vjp")

    def _sweeps(self, n_iter, n_inner, omega, shift, local, step=0.25, pivot=False):
        a = self.level_args()
        flags = self._flags.data_ptr() if local else None
        anyact = self._any_active.data_ptr() if local else None
        N.check(self._lib.glide_vanka_sweeps_ex(C.byref(a), self.f_u.data_ptr(), self.f_v.data_ptr(),
                                                self.f_H.data_ptr(), int(n_iter), int(n_inner), float(step),
                                                float(omega), float(shift), int(bool(pivot)), flags, anyact,
                                                self._scratch.data_ptr(), self._s()), "vanka")

    def vanka_smooth(self, color=0, omega=1.0, n_inner=1, shift=1.0):
        """One ``vanka_smooth`` launch: adds the face/cell deltas into
        delta_U without touching U (glide/grid.py:256-269)."""
        saved = self.U.clone()
        self._sweeps(1, n_inner, 1.0, shift, False)
        self.delta_U += self.U - saved
        self.U.copy_(saved)

    def vanka_smooth_local(self, color=0, omega=1.0, n_inner=1, shift=1.0):
        """As ``vanka_smooth`` but gated by ``error_mask`` (glide/grid.py:271-284)."""
        self.update_tile_flags()
        saved = self.U.clone()
        self._sweeps(1, n_inner, 1.0, shift, True)
        self.delta_U += self.U - saved
        self.U.copy_(saved)

    def update_tile_flags(self):
        a = self.level_args()
        N.check(self._lib.glide_tile_flags(C.byref(a), self.error_mask.data_ptr(), self._flags.data_ptr(),
                                           self._any_active.data_ptr(), self._s()), "tile flags")

    def vanka_sweep(self, n_iter, n_inner=10, omega=0.5, shift=1.0, step=0.25, pivot=False):
        """n_iter sweeps with U += omega*delta (glide/grid.py:305-310); ``step``
        is the local Newton step fraction (reference 0.25), ``pivot`` selects
        row-pivoted local solves."""
        self._sweeps(n_iter, n_inner, omega, shift, False, step, pivot)

    def vanka_sweep_local(self, n_iter, n_inner=10, omega=0.5, shift=1.0, step=0.25):
        """Sweeps gated by error_mask (glide/grid.py:312-317)."""
        self.update_tile_flags()
        self._sweeps(n_iter, n_inner, omega, shift, True, step)

    def vanka_lu(self, shift=1.0):
        """Factor every cell's local Vanka matrix at the current state with
        right-hand side f (for linear sweeps); the factors stay in this grid
        until the next call."""
        if getattr(self, "_lu", None) is None:
            self._lu = torch.empty(25 * self.nb * self.nh, dtype=self.dtype, device=self.device)
        a = self.level_args()
        N.check(self._lib.glide_vanka_lu(C.byref(a), self.f_H.data_ptr(), self._lu.data_ptr(), float(shift),
                                         self._s()), "vanka lu")

    def vanka_linear_sweep(self, rho, d, omega=0.5):
        """d += omega * additive linear Vanka update for the linear residual
        rho = r + J d (rho, d: monolithic vectors like U)."""
        ru, rv, rH = self._vec_to_fields(rho)
        du, dv, dH = self._vec_to_fields(d)
        a = self.level_args()
        N.check(self._lib.glide_vanka_linear(C.byref(a), ru.data_ptr(), rv.data_ptr(), rH.data_ptr(),
                                             self._lu.data_ptr(), du.data_ptr(), dv.data_ptr(), dH.data_ptr(),
                                             float(omega), self._scratch.data_ptr(), self._s()), "vanka linear")

    def vanka_smooth_adjoint(self, color, omega=0.5):
        """One adjoint colour update from the current r_adj (glide/grid.py:286-303)."""
        a = self.level_args()
        N.check(self._lib.glide_vanka_adjoint(C.byref(a), self.lambda_u.data_ptr(), self.lambda_v.data_ptr(),
                                              self.lambda_H.data_ptr(), self.r_adj_u.data_ptr(),
                                              self.r_adj_v.data_ptr(), self.r_adj_H.data_ptr(), int(color),
                                              float(omega), self._s()), "vanka adjoint")

    def compute_adjoint_residual(self, exact_boundary=False):
        """r_adj = f_adj - Lambda^T J."""
        a = self.level_args()
        N.check(self._lib.glide_vjp(C.byref(a), self.lambda_u.data_ptr(), self.lambda_v.data_ptr(),
                                    self.lambda_H.data_ptr(), self.f_adj_u.data_ptr(), self.f_adj_v.data_ptr(),
                                    self.f_adj_H.data_ptr(), self.r_adj_u.data_ptr(), self.r_adj_v.data_ptr(),
                                    self.r_adj_H.data_ptr(), int(exact_boundary), self._s()), "adjoint residual")

    def vanka_sweep_adjoint(self, n_iter, omega=0.5, exact_boundary=False):
        """glide/grid.py:319-330."""
        for _ in range(n_iter):
            for color in (0, 1):
                self.compute_adjoint_residual(exact_boundary)
                self.vanka_smooth_adjoint(color, omega)

    def compute_mask(self, tol=1e-1):
        """mask = H <= gamma + tol (glide/grid.py:332-334)."""
        N.check(self._lib.glide_mask_le(self.code, self.mask.data_ptr(), self.H.data_ptr(), self.gamma.data_ptr(),
                                        float(tol), self.nb * self.nh, self._s()), "mask")

    def compute_grad_beta(self, exact_boundary=False, mask_tol=1e-1):
        """grad_beta from the current Lambda (glide/grid.py:336-355)."""
        grad = self._cells()
        self.compute_mask(mask_tol)
        a = self.level_args()
        N.check(self._lib.glide_grad_beta(C.byref(a), self.lambda_u.data_ptr(), self.lambda_v.data_ptr(),
                                          grad.data_ptr(), int(exact_boundary), self._s()), "grad beta")
        self.mask.zero_()
        return grad

    def residual_norms(self):
        """Device FP64 sums of squares (r_u, r_v, FB(r_H, H-gamma)) of the
        current r (no host synchronisation)."""
        N.check(self._lib.glide_norms(self.code, self._norm_out.data_ptr(), self._norm_parts.data_ptr(),
                                      self.r_u.data_ptr(), self.r_v.data_ptr(), self.r_H.data_ptr(),
                                      self.H.data_ptr(), self.gamma.data_ptr(), self.nb * self.nu,
                                      self.nb * self.nv, self.nb * self.nh, self._s()), "norms")
        return self._norm_out
