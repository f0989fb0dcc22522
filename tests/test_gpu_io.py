"""Asynchronous VTI snapshots of device fields: a field overwritten on the
producing stream right after ``write_step`` is written with the values it had
at the call."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_snapshot_holds_values_at_the_call(tmp_path):
    from glide_b200.io import VTIWriter, read_vti
    H = torch.rand(64, 96, dtype=torch.float64, device="cuda") * 1000
    u = torch.randn(64, 96, device="cuda")
    want_H, want_u = H.float().cpu().numpy(), u.cpu().numpy()
    with VTIWriter(tmp_path, dx=1000.0) as w:
        w.write_step(0, 0.0, {"H": H, "vel": [u, u]})
        H.fill_(-1.0)
        u.mul_(0.0)
    got = read_vti(tmp_path / "output_0000.vti")
    assert np.array_equal(got["H"], np.flip(want_H, 0))
    assert np.array_equal(got["vel"][..., 0], np.flip(want_u, 0))
