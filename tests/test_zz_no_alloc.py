"""glide_vanka_sweeps_noalloc: Vanka sweeps for callers that cannot allocate.

Some callers cannot call cudaMalloc (a host framework whose memory pool owns
the device memory and hands a plugin only its inputs and outputs, or a loop
that must not pay cudaMalloc's implicit device synchronisation).  The
no-allocation entry point keeps its scratch in a fixed array inside the
library.  This test calls it through the C ABI and checks its output against
the allocating entry point (glide_vanka_sweeps with a caller-allocated
scratch) on two calls in a row, within the tolerance of the other Vanka
tests (FP64 1e-10, FP32 2e-5, norm-wise relative; the two paths run the same
kernels, so the results are expected to be identical), and that a problem
larger than the fixed array is rejected.  The file name sorts last so a run
that stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import random_state

pytestmark = pytest.mark.gpu

TOL = {torch.float64: 1e-10, torch.float32: 2e-5}


def _lib():
    from glide_b200 import _native as N
    return N.load()


def _grid(st, dtype):
    from glide_b200.grid import Grid
    ny, nx = st["H"].shape
    g = Grid(ny, nx, st["dx"], dt=st["dt"], dtype=dtype)
    for k in ("u", "v", "H", "bed", "B", "beta", "mask", "gamma", "f_u", "f_v", "f_H"):
        getattr(g, k).copy_(torch.as_tensor(st[k]))
    g.u.mul_(0.02)
    g.v.mul_(0.02)
    return g


def _rel(a, b):
    return (torch.linalg.norm((a - b).double()) / torch.linalg.norm(b.double()).clamp_min(1e-300)).item()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_matches_allocating_sweeps_twice(dtype):
    lib = _lib()
    st = random_state(n=48, seed=31)
    a_grid, b_grid = _grid(st, dtype), _grid(st, dtype)
    s = torch.cuda.current_stream().cuda_stream
    scratch = torch.empty(5 * 48 * 48, dtype=dtype, device="cuda")   # the allocating entry point's scratch
    for call in range(2):
        a_args = a_grid.level_args()
        rc = lib.glide_vanka_sweeps(C.byref(a_args), a_grid.f_u.data_ptr(), a_grid.f_v.data_ptr(),
                                    a_grid.f_H.data_ptr(), 3, 10, 0.5, 1.0, None, None, scratch.data_ptr(), s)
        assert rc == 0
        args = b_grid.level_args()
        rc = lib.glide_vanka_sweeps_noalloc(C.byref(args), b_grid.f_u.data_ptr(), b_grid.f_v.data_ptr(),
                                            b_grid.f_H.data_ptr(), 3, 10, 0.5, 1.0, None, None, s)
        assert rc == 0
        torch.cuda.synchronize()
        for x, y in ((b_grid.u, a_grid.u), (b_grid.v, a_grid.v), (b_grid.H, a_grid.H)):
            assert _rel(x, y) <= TOL[dtype], f"call {call}"


def test_noalloc_rejects_problems_beyond_its_array():
    lib = _lib()
    st = random_state(n=16, seed=32)
    g = _grid(st, torch.float64)
    args = g.level_args()
    cap_cells = lib.glide_noalloc_scratch_bytes() // (5 * 8)
    args.ny = args.nx = int(np.ceil(np.sqrt(cap_cells))) + 1   # sizes only; rejected before any launch
    rc = lib.glide_vanka_sweeps_noalloc(C.byref(args), g.f_u.data_ptr(), g.f_v.data_ptr(), g.f_H.data_ptr(), 1, 10,
                                        0.5, 1.0, None, None, torch.cuda.current_stream().cuda_stream)
    assert rc == -5   # GLIDE_E_TOO_LARGE
