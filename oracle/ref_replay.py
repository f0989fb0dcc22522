"""Replay of the reference's Python driver over the reference's own kernels.

Test infrastructure only (the FP32 GPU oracle).  ``oracle/_ref/libglide_ref.so``
holds the reference CUDA kernels compiled from the reference tree
(``oracle/build_ref.py``); this module restates the call sequences of
glide/grid.py:190-355 and glide/solver.py:71-220 around them with torch
float32 buffers, so the reference path can run where CuPy is absent.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np
import torch

LIB = Path(__file__).resolve().parent / "_ref" / "libglide_ref.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(f"{LIB} missing: build it with oracle/build_ref.py where the reference tree exists")
        L = C.CDLL(str(LIB))
        vp, i, f = C.c_void_p, C.c_int, C.c_float
        L.ref_compute_residual.argtypes = [vp] * 14 + [vp, f, f, i, i, vp]
        L.ref_compute_jvp.argtypes = [vp] * 14 + [vp, f, f, i, i, vp]
        L.ref_compute_vjp.argtypes = [vp] * 14 + [vp, f, f, i, i, vp]
        L.ref_vanka_smooth.argtypes = [vp] * 14 + [vp, f, f, i, i, i, i, f, i, vp]
        L.ref_vanka_smooth_adjoint.argtypes = [vp] * 17 + [vp, f, f, i, i, i, f, vp]
        L.ref_compute_grad_beta.argtypes = [vp] * 12 + [vp, f, f, i, i, vp]
        L.ref_transfer.argtypes = [i, vp, vp, i, i, vp]
        for n in ("ref_compute_residual", "ref_compute_jvp", "ref_compute_vjp", "ref_vanka_smooth",
                  "ref_vanka_smooth_adjoint", "ref_compute_grad_beta", "ref_transfer"):
            getattr(L, n).restype = C.c_int
        _lib = L
    return _lib


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: CUDA error {rc}")


def _s():
    return torch.cuda.current_stream().cuda_stream


def _p(t):
    return t.data_ptr()


def make_params(n=3.0, eps_reg=1e-5, water_drag=1e-3, calving_rate=1.0, gl_sigmoid_c=0.1, gl_derivatives=False):
    """5 float32 + 1 int32, as glide/kernels.py:39-49 packs them."""
    b = np.zeros(6, np.float32)
    b[:5] = [n, eps_reg, water_drag, calving_rate, gl_sigmoid_c]
    raw = b.tobytes()[:20] + np.array([int(gl_derivatives)], np.int32).tobytes()
    return torch.tensor(np.frombuffer(raw, np.uint8).copy(), device="cuda")


def transfer(op, src, dst, a, b):
    _chk(lib().ref_transfer(op, _p(src), _p(dst), a, b, _s()), f"transfer {op}")
    return dst


class RefGrid:
    """glide/grid.py:14-355 restated over torch float32 buffers."""

    def __init__(self, ny, nx, dx, dt=1.0, n=3.0, eps_reg=1e-5, water_drag=1e-3, calving_rate=1.0,
                 gl_sigmoid_c=0.1, gl_derivatives=False):
        self.ny, self.nx, self.dx, self.dt = ny, nx, float(np.float32(dx)), float(np.float32(dt))
        self.child = None
        self._kw = dict(n=n, eps_reg=eps_reg, water_drag=water_drag, calving_rate=calving_rate)
        self.params = make_params(n, eps_reg, water_drag, calving_rate, gl_sigmoid_c, gl_derivatives)
        self.nu, self.nv, self.nh = ny * (nx + 1), (ny + 1) * nx, ny * nx
        self.n_total = self.nu + self.nv + self.nh
        z = lambda: torch.zeros(self.n_total, dtype=torch.float32, device="cuda")
        for name, parts in (("U", "u v H"), ("delta_U", "delta_u delta_v delta_H"), ("Lambda", "lambda_u lambda_v lambda_H"),
                            ("Lambda_out", "lambda_u_out lambda_v_out lambda_H_out"), ("f", "f_u f_v f_H"),
                            ("f_adj", "f_adj_u f_adj_v f_adj_H"), ("F", "F_u F_v F_H"), ("Z", "Z_u Z_v Z_H"),
                            ("r", "r_u r_v r_H"), ("r_adj", "r_adj_u r_adj_v r_adj_H"), ("j", "j_u j_v j_H"),
                            ("d_U", "d_u d_v d_H"), ("l", "l_u l_v l_H"), ("w", "w_u w_v w_H"), ("y", "y_u y_v y_H"),
                            ("z", "z_u z_v z_H")):
            vec = z()
            setattr(self, name, vec)
            for pn, view in zip(parts.split(), self._views(vec)):
                setattr(self, pn, view)
        for name in ("H_prev", "chi", "phi", "bed", "beta", "B", "smb", "mask", "error_mask", "gamma"):
            setattr(self, name, torch.zeros((ny, nx), dtype=torch.float32, device="cuda"))

    def _views(self, x):
        ny, nx = self.ny, self.nx
        return (x[:self.nu].view(ny, nx + 1), x[self.nu:self.nu + self.nv].view(ny + 1, nx),
                x[self.nu + self.nv:].view(ny, nx))

    def spawn_child(self):
        self.child = RefGrid(self.ny // 2, self.nx // 2, self.dx * 2, self.dt, **self._kw)
        return self.child

    def _geo(self):
        return (C.c_float(self.dx), C.c_float(self.dt), self.ny, self.nx)

    def compute_residual(self, return_fischer_burmeister=False):
        _chk(lib().ref_compute_residual(_p(self.r_u), _p(self.r_v), _p(self.r_H), _p(self.u), _p(self.v),
                                        _p(self.H), _p(self.f_u), _p(self.f_v), _p(self.f_H), _p(self.bed),
                                        _p(self.B), _p(self.beta), _p(self.mask), _p(self.gamma), _p(self.params),
                                        *self._geo(), _s()), "residual")
        if return_fischer_burmeister:
            a, b = self.r_H, self.H - self.gamma
            return a + b - torch.sqrt(a ** 2 + b ** 2)

    def compute_F(self):
        _chk(lib().ref_compute_residual(_p(self.F_u), _p(self.F_v), _p(self.F_H), _p(self.u), _p(self.v),
                                        _p(self.H), _p(self.Z_u), _p(self.Z_v), _p(self.Z_H), _p(self.bed),
                                        _p(self.B), _p(self.beta), _p(self.mask), _p(self.gamma), _p(self.params),
                                        *self._geo(), _s()), "F")

    def compute_jvp(self):
        _chk(lib().ref_compute_jvp(_p(self.j_u), _p(self.j_v), _p(self.j_H), _p(self.u), _p(self.v), _p(self.H),
                                   _p(self.d_u), _p(self.d_v), _p(self.d_H), _p(self.bed), _p(self.B),
                                   _p(self.beta), _p(self.mask), _p(self.gamma), _p(self.params), *self._geo(),
                                   _s()), "jvp")

    def compute_vjp(self):
        self.l.zero_()
        _chk(lib().ref_compute_vjp(_p(self.l_u), _p(self.l_v), _p(self.l_H), _p(self.u), _p(self.v), _p(self.H),
                                   _p(self.lambda_u), _p(self.lambda_v), _p(self.lambda_H), _p(self.bed),
                                   _p(self.B), _p(self.beta), _p(self.mask), _p(self.gamma), _p(self.params),
                                   *self._geo(), _s()), "vjp")

    def _vanka(self, local, n_inner):
        m = self.error_mask if local else self.mask
        _chk(lib().ref_vanka_smooth(_p(self.delta_u), _p(self.delta_v), _p(self.delta_H), _p(m), _p(self.u),
                                    _p(self.v), _p(self.H), _p(self.f_u), _p(self.f_v), _p(self.f_H), _p(self.bed),
                                    _p(self.B), _p(self.beta), _p(self.gamma), _p(self.params), *self._geo(), 0,
                                    n_inner, C.c_float(1.0), int(local), _s()), "vanka")

    def vanka_sweep(self, n_iter, n_inner=10, omega=0.5):
        for _ in range(n_iter):
            self.delta_U.zero_()
            self._vanka(False, n_inner)
            self.U += np.float32(omega) * self.delta_U

    def vanka_sweep_local(self, n_iter, n_inner=10, omega=0.5):
        for _ in range(n_iter):
            self.delta_U.zero_()
            self._vanka(True, n_inner)
            self.U += np.float32(omega) * self.delta_U

    def vanka_smooth_adjoint(self, color, omega=0.5):
        self.Lambda_out.copy_(self.Lambda)
        _chk(lib().ref_vanka_smooth_adjoint(_p(self.lambda_u_out), _p(self.lambda_v_out), _p(self.lambda_H_out),
                                            _p(self.lambda_u), _p(self.lambda_v), _p(self.lambda_H), _p(self.mask),
                                            _p(self.r_adj_u), _p(self.r_adj_v), _p(self.r_adj_H), _p(self.u),
                                            _p(self.v), _p(self.H), _p(self.bed), _p(self.B), _p(self.beta),
                                            _p(self.gamma), _p(self.params), *self._geo(), color, C.c_float(omega),
                                            _s()), "vanka adjoint")
        self.Lambda.copy_(self.Lambda_out)

    def vanka_sweep_adjoint(self, n_iter, omega=0.5):
        for _ in range(n_iter):
            for color in (0, 1):
                self.r_adj.copy_(self.f_adj)
                self.compute_vjp()
                self.r_adj -= self.l
                self.vanka_smooth_adjoint(color, omega=omega)

    def compute_mask(self, tol=1e-1):
        self.mask.copy_((self.H <= (self.gamma + np.float32(tol))).float())

    def compute_grad_beta(self):
        grad = torch.zeros((self.ny, self.nx), dtype=torch.float32, device="cuda")
        self.compute_mask()
        _chk(lib().ref_compute_grad_beta(_p(grad), _p(self.u), _p(self.v), _p(self.H), _p(self.lambda_u),
                                         _p(self.lambda_v), _p(self.lambda_H), _p(self.bed), _p(self.B),
                                         _p(self.beta), _p(self.mask), _p(self.gamma), _p(self.params), *self._geo(),
                                         _s()), "grad")
        self.mask.zero_()
        return grad


# transfer wrappers (glide/kernels.py:90-236)
def restrict_vfacet(uf, uc):
    return transfer(0, uf, uc, uc.shape[0], uc.shape[1] - 1)


def restrict_hfacet(vf, vc):
    return transfer(1, vf, vc, vc.shape[0] - 1, vc.shape[1])


def restrict_cell_centered(hf, hc):
    return transfer(2, hf, hc, hc.shape[0], hc.shape[1])


def restrict_max_pool(hf, hc):
    return transfer(3, hf, hc, hc.shape[0], hc.shape[1])


def prolongate_vfacet(uc, uf, smooth=True):
    return transfer(7 if smooth else 4, uc, uf, uf.shape[0], uf.shape[1] - 1)


def prolongate_hfacet(vc, vf, smooth=True):
    return transfer(8 if smooth else 5, vc, vf, vf.shape[0] - 1, vf.shape[1])


def prolongate_cell_centered(hc, hf, smooth=True):
    return transfer(9 if smooth else 6, hc, hf, hf.shape[0], hf.shape[1])


def restrict_parameters(g):
    c = g.child
    for name in ("bed", "B", "beta", "H_prev", "smb"):
        restrict_cell_centered(getattr(g, name), getattr(c, name))


def restrict_parameters_to_hierarchy(g):
    while g.child is not None:
        restrict_parameters(g)
        g = g.child


def fascd_vcycle(grid, thklim, finest=False):
    """glide/solver.py:71-157, step for step."""
    thk = np.float32(thklim)
    if finest:
        grid.w.copy_(grid.U)
        grid.chi.copy_(grid.gamma - grid.H)
    if grid.child is None:
        grid.gamma.copy_(grid.w_H + grid.chi)
        grid.vanka_sweep(200)
        grid.gamma.fill_(float(thk))
        return
    c = grid.child
    restrict_max_pool(grid.chi, c.chi)
    prolongate_cell_centered(-c.chi, grid.phi, smooth=False)
    grid.phi += grid.chi
    grid.gamma.copy_(grid.w_H + grid.phi)
    grid.vanka_sweep(10)
    grid.gamma.fill_(float(thk))
    grid.y.copy_(grid.U - grid.w)
    restrict_vfacet(grid.u, c.u)
    restrict_hfacet(grid.v, c.v)
    restrict_cell_centered(grid.H, c.H)
    c.w.copy_(c.U)
    grid.compute_residual()
    restrict_vfacet(grid.r_u, c.r_u)
    restrict_hfacet(grid.r_v, c.r_v)
    restrict_cell_centered(grid.r_H, c.r_H)
    c.compute_F()
    c.f.copy_(c.F - c.r)
    fascd_vcycle(c, thklim)
    c.z.copy_(c.U - c.w)
    prolongate_vfacet(c.z_u, grid.z_u)
    prolongate_hfacet(c.z_v, grid.z_v)
    prolongate_cell_centered(c.z_H, grid.z_H, smooth=False)
    grid.z += grid.y
    grid.U.copy_(grid.w + grid.z)
    grid.gamma.copy_(grid.w_H + grid.chi)
    grid.vanka_sweep(10)
    for _ in range(10):
        grid.compute_residual()
        a = grid.r_H
        b = grid.H - grid.gamma
        rss = a + b - torch.sqrt(a ** 2 + b ** 2)
        tot = (grid.r_u[:, 1:].abs() + grid.r_u[:, :-1].abs() + grid.r_v[1:].abs() + grid.r_v[:-1].abs() + rss.abs())
        grid.error_mask.copy_((tot > np.float32(0.01)).float())
        grid.vanka_sweep_local(10)
    grid.gamma.fill_(float(thk))


def adjoint_vcycle(grid):
    """glide/solver.py:160-220, step for step."""
    if grid.child is None:
        grid.compute_mask()
        grid.vanka_sweep_adjoint(100, omega=1.0)
        grid.mask.zero_()
        return
    grid.compute_mask()
    grid.vanka_sweep_adjoint(10, omega=1.0)
    grid.mask.zero_()
    grid.r_adj.copy_(grid.f_adj)
    grid.compute_vjp()
    grid.r_adj -= grid.l
    c = grid.child
    restrict_vfacet(grid.lambda_u, c.lambda_u)
    restrict_hfacet(grid.lambda_v, c.lambda_v)
    restrict_cell_centered(grid.lambda_H, c.lambda_H)
    restrict_parameters(grid)
    c.f_adj.zero_()
    restrict_vfacet(grid.r_adj_u, c.f_adj_u)
    restrict_hfacet(grid.r_adj_v, c.f_adj_v)
    restrict_cell_centered(grid.r_adj_H, c.f_adj_H)
    c.Lambda.zero_()
    c.Lambda_out.zero_()
    adjoint_vcycle(c)
    grid.z.zero_()
    prolongate_vfacet(c.lambda_u, grid.z_u)
    prolongate_hfacet(c.lambda_v, grid.z_v)
    prolongate_cell_centered(c.lambda_H, grid.z_H, smooth=True)
    grid.lambda_u += grid.z_u
    grid.lambda_v += grid.z_v
    grid.lambda_H += grid.z_H
    grid.compute_mask()
    grid.vanka_sweep_adjoint(10, omega=1.0)
    grid.mask.zero_()


class RefIcePhysics:
    """glide/physics.py:49-242 over the reference kernels."""

    def __init__(self, ny, nx, dx, n_levels=5, n=3.0, eps_reg=1e-5, thklim=0.1, water_drag=1e-3,
                 calving_rate=1.0, gl_sigmoid_c=0.1, gl_derivatives=False):
        self.thklim = float(np.float32(thklim))
        self.grid = RefGrid(ny, nx, dx, 1.0, n, eps_reg, water_drag, calving_rate, gl_sigmoid_c, gl_derivatives)
        self.grids = [self.grid]
        for _ in range(n_levels - 1):
            self.grids.append(self.grids[-1].spawn_child())

    def set_geometry(self, bed, thickness):
        g = self.grid
        g.bed.copy_(torch.as_tensor(np.asarray(bed, np.float32)))
        g.H.copy_(torch.as_tensor(np.asarray(thickness, np.float32)))
        g.H_prev.copy_(g.H)
        g.gamma.fill_(self.thklim)
        for par, ch in zip(self.grids[:-1], self.grids[1:]):
            restrict_cell_centered(par.bed, ch.bed)
            restrict_cell_centered(par.H, ch.H)
            restrict_cell_centered(par.H_prev, ch.H_prev)
            ch.gamma.fill_(self.thklim)

    def set_parameters(self, B=None, beta=None, smb=None):
        g = self.grid
        if B is not None:
            Bn = np.asarray(B, np.float32)
            if Bn.ndim == 0:
                g.B.fill_(float(Bn))
            else:
                g.B.copy_(torch.as_tensor(Bn))
        if beta is not None:
            g.beta.copy_(torch.as_tensor(np.asarray(beta, np.float32)))
        if smb is not None:
            g.smb.copy_(torch.as_tensor(np.asarray(smb, np.float32)))
        restrict_parameters_to_hierarchy(g)

    def residual_norm(self):
        g = self.grid
        rss = g.compute_residual(return_fischer_burmeister=True)
        return float(torch.sqrt(torch.linalg.norm(g.r_u) ** 2 + torch.linalg.norm(g.r_v) ** 2
                                + torch.linalg.norm(rss) ** 2))

    def forward(self, dt, n_vcycles=3, update_geometry=True, history=None):
        for g in self.grids:
            g.dt = float(np.float32(dt))
        g = self.grid
        g.f_H.copy_(g.H_prev / np.float32(g.dt) + g.smb)
        r0 = self.residual_norm() if history is not None else None
        for _ in range(n_vcycles):
            fascd_vcycle(g, self.thklim, finest=True)
            if history is not None:
                history.append(self.residual_norm() / r0)
        if update_geometry:
            g.H_prev.copy_(g.H)
        return g.u, g.v, g.H

    def adjoint(self, dL_du, dL_dv, dL_dH, n_vcycles=2):
        g = self.grid
        g.f_adj_u.copy_(-torch.as_tensor(np.asarray(dL_du, np.float32)))
        g.f_adj_v.copy_(-torch.as_tensor(np.asarray(dL_dv, np.float32)))
        g.f_adj_H.copy_(-torch.as_tensor(np.asarray(dL_dH, np.float32)))
        g.Lambda.zero_()
        g.Lambda_out.zero_()
        for _ in range(n_vcycles):
            adjoint_vcycle(g)
        return g.compute_grad_beta()
