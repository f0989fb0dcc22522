import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the native library")
    config.addinivalue_line("markers", "slow: long-running")


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_ok():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def random_state(n=32, seed=0, dx=10000.0, vel=50.0, mask_frac=0.2):
    """Seeded inputs for single-operator parity: the dome geometry with random
    velocities, a random active-set mask and random tangents."""
    from glide_b200.synthetic import dome_case
    c = dome_case(seed, n=n, dx=dx)
    rng = np.random.default_rng(seed + 100)
    ny = nx = n
    st = dict(
        u=rng.standard_normal((ny, nx + 1)) * vel, v=rng.standard_normal((ny + 1, nx)) * vel,
        H=c.thickness + rng.random((ny, nx)) * 5.0, bed=c.bed, B=c.B, beta=c.beta,
        mask=(rng.random((ny, nx)) < mask_frac).astype(float), gamma=np.full((ny, nx), 0.1),
        f_u=rng.standard_normal((ny, nx + 1)), f_v=rng.standard_normal((ny + 1, nx)),
        f_H=rng.standard_normal((ny, nx)),
        d_u=rng.standard_normal((ny, nx + 1)), d_v=rng.standard_normal((ny + 1, nx)), d_H=rng.standard_normal((ny, nx)),
        dx=c.dx, dt=10.0)
    return st
