"""glide_vanka_sweeps_noalloc: Vanka sweeps for callers that cannot allocate.

Some callers cannot call cudaMalloc (a host framework whose memory pool owns
the device memory and hands a plugin only its inputs and outputs, or a loop
that must not pay cudaMalloc's implicit device synchronisation).  The
no-allocation entry point keeps its scratch in a fixed array inside the
library.  This test calls it through the C ABI and checks its output against
the allocating entry point (glide_vanka_sweeps with a caller-allocated
scratch) on two calls in a row, for full sweeps and for sweeps gated by the
error-indicator tile flags (the local path).  Both entry points run the same
kernels on the same inputs, so the results must be bit-identical (the other
Vanka tests' tolerances, FP64 1e-10 and FP32 2e-5, are the looser bound this
implies).  The second call must not change the device memory in use, and a
problem larger than the fixed array is rejected.  The file name sorts last so
a run that stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import random_state

pytestmark = pytest.mark.gpu


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
    g.mask.zero_()
    return g


def _local_flags(lib, g, s):
    """Error mask and tile flags of the grid's residual, threshold at the
    median indicator, so that part of the tiles is active."""
    g.compute_residual()
    fb = g.r_H + (g.H - g.gamma) - torch.sqrt(g.r_H ** 2 + (g.H - g.gamma) ** 2)
    ind = (g.r_u[:, 1:].abs() + g.r_u[:, :-1].abs() + g.r_v[1:].abs() + g.r_v[:-1].abs() + fb.abs())
    thr = float(ind.double().median())
    a = g.level_args()
    rc = lib.glide_error_mask(C.byref(a), g.r_u.data_ptr(), g.r_v.data_ptr(), g.r_H.data_ptr(), thr,
                              g.error_mask.data_ptr(), g._flags.data_ptr(), g._any_active.data_ptr(), s)
    assert rc == 0
    torch.cuda.synchronize()
    frac = float(g.error_mask.double().mean())
    assert 0.05 < frac < 0.95, frac
    return g._flags.data_ptr(), g._any_active.data_ptr()


@pytest.mark.parametrize("local", [False, True], ids=["full", "local"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_matches_allocating_sweeps_twice(dtype, local):
    lib = _lib()
    st = random_state(n=48, seed=31)
    a_grid, b_grid = _grid(st, dtype), _grid(st, dtype)
    s = torch.cuda.current_stream().cuda_stream
    scratch = torch.empty(5 * 48 * 48, dtype=dtype, device="cuda")   # the allocating entry point's scratch
    a_flags = _local_flags(lib, a_grid, s) if local else (None, None)
    b_flags = _local_flags(lib, b_grid, s) if local else (None, None)
    for call in range(2):
        a_args = a_grid.level_args()
        rc = lib.glide_vanka_sweeps(C.byref(a_args), a_grid.f_u.data_ptr(), a_grid.f_v.data_ptr(),
                                    a_grid.f_H.data_ptr(), 3, 10, 0.5, 1.0, a_flags[0], a_flags[1],
                                    scratch.data_ptr(), s)
        assert rc == 0
        args = b_grid.level_args()
        torch.cuda.synchronize()
        used0, free0 = torch.cuda.memory_allocated(), torch.cuda.mem_get_info()[0]
        rc = lib.glide_vanka_sweeps_noalloc(C.byref(args), b_grid.f_u.data_ptr(), b_grid.f_v.data_ptr(),
                                            b_grid.f_H.data_ptr(), 3, 10, 0.5, 1.0, b_flags[0], b_flags[1], s)
        assert rc == 0
        torch.cuda.synchronize()
        if call == 1:   # the first call may load kernels lazily; the second allocates nothing at all
            assert torch.cuda.memory_allocated() == used0
            assert torch.cuda.mem_get_info()[0] == free0
        for x, y in ((b_grid.u, a_grid.u), (b_grid.v, a_grid.v), (b_grid.H, a_grid.H)):
            assert torch.equal(x, y), f"call {call}"
        assert not torch.equal(a_grid.u, torch.as_tensor(st["u"], dtype=dtype, device="cuda") * 0.02)


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
