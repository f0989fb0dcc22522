"""Seeded synthetic geometries standing in for the reference's real datasets.

The reference drives its solver with BedMachine / MAR / velocity mosaics
(glide/data.py:23-27), which are not available here.  These generators build
seeded inputs with the shapes, resolutions and value ranges of the workloads
this package is measured on.  All fields are returned as float64 NumPy arrays
in the reference's "head" units: stresses divided by rho_i*g, velocities in
m/a, time in years (examples/greenland/greenland_forward.py:90-91).

Unit conversions (Pa -> head units):
    B_head    = B[Pa s^(1/3)] * (3.156e7 s/a)^(-1/3) / (917*9.81)
    beta_head = beta[Pa a/m] / (917*9.81)
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

RHO_I = 917.0
RHO_W = 1000.0
G = 9.81
SEC_PER_YEAR = 3.156e7
RHO_G = RHO_I * G


def B_head(B_pa_s13: float) -> float:
    return B_pa_s13 * SEC_PER_YEAR ** (-1.0 / 3.0) / RHO_G


def beta_head(beta_pa_a_m):
    return np.asarray(beta_pa_a_m) / RHO_G


@dataclass
class Case:
    """One synthetic problem: geometry, parameters and solver settings."""
    name: str
    ny: int
    nx: int
    dx: float
    n_levels: int
    bed: np.ndarray
    thickness: np.ndarray
    B: np.ndarray
    beta: np.ndarray
    smb: np.ndarray
    dt: float = 10.0
    thklim: float = 0.1
    kwargs: dict = field(default_factory=dict)   # extra IcePhysics kwargs
    info: dict = field(default_factory=dict)     # recorded generator choices


def _grf(rng, ny, nx, dx, corr_len):
    """Zero-mean unit-variance Gaussian random field with a Gaussian
    covariance of correlation length ``corr_len`` (metres)."""
    w = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny, d=dx)[:, None] * 2 * np.pi
    kx = np.fft.fftfreq(nx, d=dx)[None, :] * 2 * np.pi
    filt = np.exp(-0.25 * (kx ** 2 + ky ** 2) * corr_len ** 2)
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    s = f.std()
    return f / s if s > 0 else f


def _spectral_noise(rng, ny, nx, sigma, slope=2.0):
    """Isotropic power-law noise |k|^-slope, scaled to standard deviation sigma."""
    w = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = 1.0
    amp = k ** (-slope / 1.0)
    amp[0, 0] = 0.0
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * amp))
    return sigma * f / f.std()


def _centres(ny, nx, dx):
    y = (np.arange(ny) + 0.5) * dx
    x = (np.arange(nx) + 0.5) * dx
    return y[:, None] - 0.5 * ny * dx, x[None, :] - 0.5 * nx * dx


def surface(bed, H):
    """s = H + max(bed, -0.917 H) (glide/physics.py:244-247)."""
    return H + np.maximum(bed, -RHO_I / 1000.0 * H)


def dome_case(seed=0, n=64, dx=5000.0, n_levels=3, thklim=0.1, bump_width=40e3):
    """Plain-method case: 64x64, dx=5 km, 3 levels.

    Bed: 500 m Gaussian bump of width ``bump_width`` plus power-law spectral
    noise with sigma=50 m.  Thickness: paraboloid dome, 2000 m peak, zero at
    r=140 km (plus thklim everywhere, as glide/data.py:258 does).  Glen n=3,
    B=1e8 Pa s^(1/3).  beta = 1e3*lognormal(0,0.5) Pa a/m.
    SMB = 0.5 - 1e-3*(s-1000) m/a.
    """
    rng = np.random.default_rng(seed)
    Y, X = _centres(n, n, dx)
    r2 = X ** 2 + Y ** 2
    bed = 500.0 * np.exp(-r2 / (2 * bump_width ** 2)) + _spectral_noise(rng, n, n, 50.0)
    H = 2000.0 * np.clip(1.0 - r2 / 140e3 ** 2, 0.0, None) + thklim
    beta = beta_head(1e3 * rng.lognormal(0.0, 0.5, (n, n)))
    B = np.full((n, n), B_head(1e8))
    smb = 0.5 - 1e-3 * (surface(bed, H) - 1000.0)
    return Case("dome64", n, n, dx, n_levels, bed, H, B, beta, smb, dt=10.0, thklim=thklim,
                info=dict(seed=seed, bump_width_m=bump_width, noise_sigma_m=50.0, noise="power-law |k|^-2"))


def ice_sheet_case(seed=0, n=512, dx=1500.0, n_levels=5, thklim=0.1, h_max=3000.0, n_troughs=20,
                   beta_corr=20e3, name=None):
    """Continental-scale case: elliptic dome up to ``h_max`` cut by radial
    troughs whose bed lies 300-800 m below sea level at the margins; beta is
    a log-Gaussian random field with ``beta_corr`` correlation length.
    """
    rng = np.random.default_rng(seed)
    Y, X = _centres(n, n, dx)
    L = 0.5 * n * dx
    ax, ay = 0.80 * L * rng.uniform(0.9, 1.0), 0.70 * L * rng.uniform(0.9, 1.0)
    rho = np.sqrt((X / ax) ** 2 + (Y / ay) ** 2)
    H = h_max * np.sqrt(np.clip(1.0 - rho ** 2, 0.0, None))
    theta = np.arctan2(Y, X)
    bed = 400.0 * (1.0 - rho) + _spectral_noise(rng, n, n, 60.0)
    angles = rng.uniform(-np.pi, np.pi, n_troughs)
    depths = rng.uniform(300.0, 800.0, n_troughs)
    widths = rng.uniform(0.04, 0.09, n_troughs)
    for a, d, w in zip(angles, depths, widths):
        dth = np.angle(np.exp(1j * (theta - a)))
        prof = np.exp(-0.5 * (dth / w) ** 2)
        # trough deepens towards the margin: bed -> -d at rho>=1
        bed = bed - prof * np.clip(rho, 0.0, 1.2) * (d + 400.0 * (1.0 - np.clip(rho, 0, 1)))
    H = H + thklim
    logb = np.log(1e3) + 1.0 * _grf(rng, n, n, dx, beta_corr)
    beta = beta_head(np.exp(logb))
    B = np.full((n, n), B_head(1e8))
    smb = 0.5 - 1e-3 * (surface(bed, H) - 1000.0)
    return Case(name or f"ice_sheet{n}", n, n, dx, n_levels, bed, H, B, beta, smb, dt=10.0, thklim=thklim,
                info=dict(seed=seed, h_max=h_max, n_troughs=n_troughs, beta_corr_m=beta_corr))


def continental_case(seed=0):
    """512x512, dx=1500 m, 5 levels."""
    return ice_sheet_case(seed=seed, n=512, dx=1500.0, n_levels=5, name="continental512")


def dome_sheet_case(seed=0, n=1024, dx=1000.0, n_levels=6, thklim=0.1, name=None):
    """Grounded dome family (the config-1 geometry generalised to any size).

    Paraboloid dome with a random centre offset (+-10% of the domain), radius
    30-42% of the domain width and 1500-3000 m peak; bed = 3-6 Gaussian bumps
    of +-500 m (width 1/10 of the domain) plus power-law noise (sigma 50 m);
    log beta is a Gaussian random field (20 km correlation, sigma 0.5) around
    log(1e3 Pa a/m); B = 1e8 Pa s^(1/3); SMB = 0.5 - 1e-3 (s - 1000) m/a.
    """
    rng = np.random.default_rng(seed)
    Y, X = _centres(n, n, dx)
    L = n * dx
    cy, cx = rng.uniform(-0.1, 0.1, 2) * L
    R = L * rng.uniform(0.30, 0.42)
    hmax = rng.uniform(1500.0, 3000.0)
    r2 = (X - cx) ** 2 + (Y - cy) ** 2
    H = hmax * np.clip(1.0 - r2 / R ** 2, 0.0, None) + thklim
    bed = _spectral_noise(rng, n, n, 50.0)
    for _ in range(int(rng.integers(3, 7))):
        by, bx = rng.uniform(-0.4, 0.4, 2) * L
        amp = rng.uniform(-500.0, 500.0)
        bed = bed + amp * np.exp(-((X - bx) ** 2 + (Y - by) ** 2) / (2 * (0.1 * L) ** 2))
    logb = np.log(1e3) + 0.5 * _grf(rng, n, n, dx, 20e3)
    beta = beta_head(np.exp(logb))
    B = np.full((n, n), B_head(1e8))
    smb = 0.5 - 1e-3 * (surface(bed, H) - 1000.0)
    return Case(name or f"dome_sheet{n}", n, n, dx, n_levels, bed, H, B, beta, smb, dt=10.0, thklim=thklim,
                info=dict(seed=seed, family="grounded dome", hmax=hmax, radius_m=R))


def learned_guess_case(seed=0, n=1024, dx=1000.0, n_levels=6):
    """Fresh geometry for the learned-guess workload: 1024x1024, dx=1 km, 6 levels."""
    return dome_sheet_case(seed=seed, n=n, dx=dx, n_levels=n_levels, name=f"sheet{n}")


def training_patch_case(seed, n=256, dx=1000.0, n_levels=4):
    """A 256x256 training patch (dx=1 km) from the same family."""
    return dome_sheet_case(seed=10_000 + seed, n=n, dx=dx, n_levels=n_levels, name=f"patch{n}")


def marine_case(seed=0, n=4096, dx=1000.0, n_levels=7, thklim=0.1):
    """Marine ice sheet with floating shelves: beta=0 where
    H < 1.1*(-bed)*rho_w/rho_i, H from 0 to 4000 m."""
    c = ice_sheet_case(seed=seed, n=n, dx=dx, n_levels=n_levels, thklim=thklim, h_max=4000.0, name=f"marine{n}")
    bed = c.bed - 600.0
    H = np.clip(c.thickness, thklim, 4000.0)
    floating = H < 1.1 * (-bed) * RHO_W / RHO_I
    beta = np.where(floating, 0.0, c.beta)
    smb = 0.5 - 1e-3 * (surface(bed, H) - 1000.0)
    return Case(f"marine{n}", n, n, dx, n_levels, bed, H, c.B, beta, smb, dt=10.0, thklim=thklim,
                info=dict(c.info, floating_fraction=float(floating.mean())))
