"""The other root of a cell's mass balance (the finish's branch hop), on the host.

r_H(H) = H/dt + c (1 - g(H)) H + D - f_H with g the grounding sigmoid of
bed + 0.917 H (glide/cuda/flux.cu:187-211).  With dt = 10 a, c = 1 /a and
f_H = 50 m/a (H_prev = 500 m, no SMB) a cell on a bed at -300 m has a
grounded root at 500 m and a floating root at 45.5 m (flotation: 327 m).
The roots take g as exactly 0 or 1, so what is left of r_H at a root is the
sigmoid's tail, c H min(g, 1 - g).
"""
import math

import pytest

from glide_b200.physics import RHO_ICE, other_mass_root


def _g(H, bed, sig_c=0.1):
    return 1.0 / (1.0 + math.exp(-max(min(sig_c * (bed + RHO_ICE / 1000.0 * H), 20.0), -20.0)))


def _r(H, bed, f_H, D, dt=10.0, c=1.0):
    return H / dt + c * (1.0 - _g(H, bed)) * H + D - f_H


def _tail(H, bed, c=1.0):
    g = _g(H, bed)
    return c * H * min(g, 1.0 - g) * (1.0 + 1e-9) + 1e-12


@pytest.mark.parametrize("D", [0.0, 5.0, -3.0])
def test_grounded_to_floating_and_back(D):
    bed, f_H = -300.0, 50.0
    Hg = (f_H - D) * 10.0
    Hf = (f_H - D) / 1.1
    # from the grounded root, the floating one, and back
    H1 = other_mass_root(Hg, bed, f_H, _r(Hg, bed, f_H, D), 10.0, 1.0, 0.1, 0.1)
    assert H1 == pytest.approx(Hf, rel=1e-6)
    assert abs(_r(H1, bed, f_H, D)) <= _tail(H1, bed)
    H2 = other_mass_root(Hf, bed, f_H, _r(Hf, bed, f_H, D), 10.0, 1.0, 0.1, 0.1)
    assert H2 == pytest.approx(Hg, rel=1e-6)
    assert abs(_r(H2, bed, f_H, D)) <= _tail(H2, bed)


def test_root_off_the_branch_is_refused():
    # a shallow bed: flotation thickness 11 m, below the floating root (45 m)
    assert other_mass_root(500.0, -10.0, 50.0, _r(500.0, -10.0, 50.0, 0.0), 10.0, 1.0, 0.1, 0.1) is None
    # a root at or below the thickness limit
    assert other_mass_root(500.0, -300.0, 50.0, _r(500.0, -300.0, 50.0, 49.99), 10.0, 1.0, 0.1, 0.1) is None
