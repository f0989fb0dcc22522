"""ctypes binding of the C ABI in ``include/glide_b200.h``.

The shared library is built in-tree (``python -m glide_b200.build``).  There
is no fallback: if the library or a CUDA device is missing every call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import torch

_LIB_PATH = Path(__file__).resolve().parent / "libglide_b200.so"
_lib = None

F32, F64 = 0, 1
ERRORS = {-1: "unsupported dtype", -2: "bad shape or argument", -3: "null pointer", -4: "CUDA graph failure",
          -5: "too large (a field of 2^31 elements or more, or a fixed buffer too small)"}

SYMBOLS = [
    "glide_residual", "glide_jvp", "glide_vjp", "glide_grad_beta", "glide_vanka_sweeps", "glide_vanka_cells",
    "glide_error_mask",
    "glide_tile_flags", "glide_vanka_adjoint", "glide_restrict", "glide_prolong", "glide_lincomb", "glide_fill",
    "glide_mask_le", "glide_convert", "glide_norms", "glide_norm_parts", "glide_fascd_vcycle",
    "glide_adjoint_vcycle", "glide_restrict_parameters", "glide_graph_create", "glide_graph_launch",
    "glide_graph_destroy", "glide_launch_count", "glide_version", "glide_vanka_sweeps_noalloc",
    "glide_noalloc_scratch_bytes", "glide_vanka_sweeps_ex", "glide_vanka_lu", "glide_vanka_linear",
    "glide_misfit", "glide_tikhonov", "glide_loss_parts", "glide_jvp_add",
    "glide_linear_setup", "glide_linear_vcycle", "glide_vanka_lu_masked", "glide_newton_rhs", "glide_newton_update",
    "glide_active_mask", "glide_dots", "glide_dots_parts", "glide_combine",
]


class PhysicsParams(C.Structure):
    """GlidePhysicsParams (reference PhysicsParams, glide/cuda/common.cu:240-247)."""
    _fields_ = [("n", C.c_double), ("eps_reg", C.c_double), ("water_drag", C.c_double),
                ("calving_rate", C.c_double), ("gl_sigmoid_c", C.c_double), ("gl_derivatives", C.c_int)]


class LevelArgs(C.Structure):
    _fields_ = [("ny", C.c_int), ("nx", C.c_int), ("nb", C.c_int), ("dtype", C.c_int),
                ("dx", C.c_double), ("dt", C.c_double), ("params", PhysicsParams),
                ("u", C.c_void_p), ("v", C.c_void_p), ("H", C.c_void_p),
                ("bed", C.c_void_p), ("B", C.c_void_p), ("beta", C.c_void_p),
                ("mask", C.c_void_p), ("gamma", C.c_void_p)]


class Level(C.Structure):
    _fields_ = [("a", LevelArgs),
                ("U", C.c_void_p), ("f", C.c_void_p), ("w", C.c_void_p), ("r", C.c_void_p), ("z", C.c_void_p),
                ("chi", C.c_void_p), ("err_mask", C.c_void_p),
                ("lam", C.c_void_p), ("f_adj", C.c_void_p), ("r_adj", C.c_void_p),
                ("H_prev", C.c_void_p), ("smb", C.c_void_p),
                ("scratch", C.c_void_p), ("flags", C.c_void_p), ("any_active", C.c_void_p),
                ("ls_tmp", C.c_void_p), ("ls_norms", C.c_void_p), ("norm_parts", C.c_void_p),
                ("lu", C.c_void_p), ("lin_rhs", C.c_void_p), ("lin_rho", C.c_void_p), ("lin_d", C.c_void_p),
                ("r_raw", C.c_void_p)]

LS_CANDIDATES = 4  # GLIDE_LS_CANDIDATES


class SolverConfig(C.Structure):
    _fields_ = [("thklim", C.c_double), ("n_coarse", C.c_int), ("n_smooth", C.c_int), ("n_local_outer", C.c_int),
                ("n_local", C.c_int), ("n_newton", C.c_int), ("omega", C.c_double), ("shift", C.c_double),
                ("err_threshold", C.c_double), ("adj_coarse", C.c_int), ("adj_smooth", C.c_int),
                ("adj_omega", C.c_double), ("exact_adjoint", C.c_int), ("smooth_H_correction", C.c_int),
                ("newton_step", C.c_double), ("pivoted_lu", C.c_int), ("coarse_line_search", C.c_int),
                ("lin_pre", C.c_int), ("lin_post", C.c_int), ("lin_coarse", C.c_int), ("lin_omega", C.c_double),
                ("lin_shift", C.c_double), ("adj_active_tol", C.c_double)]


class NativeError(RuntimeError):
    pass


def lib_path() -> Path:
    return _LIB_PATH


def load():
    """Load the native library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise NativeError(f"native library {_LIB_PATH} is missing; run `python -m glide_b200.build`")
    lib = C.CDLL(str(_LIB_PATH))
    vp, i, d, i64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
    LA = C.POINTER(LevelArgs)
    sig = {
        "glide_residual": [LA, vp, vp, vp, vp, vp, vp, vp],
        "glide_jvp": [LA, vp, vp, vp, vp, vp, vp, vp],
        "glide_jvp_add": [LA, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp],
        "glide_vjp": [LA, vp, vp, vp, vp, vp, vp, vp, vp, vp, i, vp],
        "glide_grad_beta": [LA, vp, vp, vp, i, vp],
        "glide_vanka_sweeps": [LA, vp, vp, vp, i, i, d, d, vp, vp, vp, vp],
        "glide_vanka_sweeps_ex": [LA, vp, vp, vp, i, i, d, d, d, i, vp, vp, vp, vp],
        "glide_vanka_lu": [LA, vp, vp, d, vp],
        "glide_misfit": [i, i, d, vp, vp, vp, vp, i64, i64, vp, vp, vp, vp, vp],
        "glide_tikhonov": [i, vp, i, i, vp, vp, vp, vp],
        "glide_loss_parts": [i64],
        "glide_vanka_linear": [LA, vp, vp, vp, vp, vp, vp, vp, d, vp, vp],
        "glide_vanka_cells": [LA, vp, vp, vp, i, i, d, vp, vp, vp, vp],
        "glide_error_mask": [LA, vp, vp, vp, d, vp, vp, vp, vp],
        "glide_tile_flags": [LA, vp, vp, vp, vp],
        "glide_vanka_adjoint": [LA, vp, vp, vp, vp, vp, vp, i, d, vp],
        "glide_restrict": [i, i, i, vp, vp, i, i, i, vp],
        "glide_prolong": [i, i, i, i, vp, vp, i, i, i, vp],
        "glide_lincomb": [i, vp, vp, d, vp, d, i64, vp],
        "glide_fill": [i, vp, d, i64, vp],
        "glide_mask_le": [i, vp, vp, vp, d, i64, vp],
        "glide_convert": [i, vp, vp, i64, i, vp],
        "glide_norms": [i, vp, vp, vp, vp, vp, vp, vp, i64, i64, i64, vp],
        "glide_norm_parts": [i64],
        "glide_fascd_vcycle": [C.POINTER(Level), i, i, i, C.POINTER(SolverConfig), vp],
        "glide_adjoint_vcycle": [C.POINTER(Level), i, i, C.POINTER(SolverConfig), vp],
        "glide_restrict_parameters": [C.POINTER(Level), i, i, vp],
        "glide_graph_create": [C.POINTER(Level), i, C.POINTER(SolverConfig), i, C.POINTER(C.c_void_p)],
        "glide_graph_launch": [vp, vp],
        "glide_graph_destroy": [vp],
        "glide_launch_count": [],
        "glide_vanka_sweeps_noalloc": [LA, vp, vp, vp, i, i, d, d, vp, vp, vp],
        "glide_noalloc_scratch_bytes": [],
        "glide_version": [],
        "glide_linear_setup": [C.POINTER(Level), i, C.POINTER(SolverConfig), vp],
        "glide_linear_vcycle": [C.POINTER(Level), i, C.POINTER(SolverConfig), vp],
        "glide_vanka_lu_masked": [LA, vp, d, vp],
        "glide_newton_rhs": [LA, vp, vp, vp, vp, i, vp],
        "glide_newton_update": [LA, vp, vp, vp, i, d, vp],
        "glide_active_mask": [LA, vp, vp, vp],
        "glide_dots": [i, i64, i, vp, i64, vp, vp, vp, vp],
        "glide_dots_parts": [i64],
        "glide_combine": [i, i64, i, vp, i64, vp, d, vp, d, vp],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = {"glide_version": C.c_char_p, "glide_launch_count": C.c_longlong,
                     "glide_noalloc_scratch_bytes": C.c_size_t}.get(name, C.c_int)
    _lib = lib
    return lib


def check(rc: int, what: str = "glide call"):
    if rc != 0:
        msg = ERRORS.get(rc) or f"CUDA error {rc}: {torch.cuda.get_device_name() if torch.cuda.is_available() else ''}"
        raise NativeError(f"{what} failed ({rc}): {msg}")


def stream_handle(stream=None) -> int:
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream


def ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


def dtype_code(dt: torch.dtype) -> int:
    if dt == torch.float32:
        return F32
    if dt == torch.float64:
        return F64
    raise NativeError(f"unsupported dtype {dt}")
