"""Seeded synthetic problems for the benchmark and the parity tests.

No dataset is involved: every input is generated here from numpy
``default_rng(seed)`` streams, identically for the oracle and the GPU.

* ``poisson_noise(n)``      5-point Poisson, b = (sin(pi x) sin(pi y) + U[-1e-3,1e-3]) h^2.
* ``hetero_diffusion(n)``   9-point bilinear-FE operator of -div(K grad u) on an
  (n+1)^2 cell mesh: K = exp(g), g a Gaussian random field (Gaussian covariance,
  correlation length ell, standard deviation sigma), optional axis-aligned
  rectangular inclusions with a contrast factor, optional anisotropy
  (ky = eps * kx in cells whose centre has y > 0.5); b = U[0,1] h^2.
* ``hetero3_coefficients(n)`` / ``hetero3_rhs(n)``  3D lognormal cell coefficient
  (Gaussian field, correlation length 1/16, sigma 1.5, periodic synthesis box)
  with 16 boxes of contrast 1e3; b = U[-1,1] h^3.
"""
import math

import numpy as np

from . import gallery


def poisson_noise(n, seed=0):
    """5-point Poisson, n x n interior nodes, h = 1/(n+1)."""
    so = gallery.poisson(n, n)
    h = 1.0 / (n + 1)
    x = np.arange(1, n + 1) * h
    f = np.sin(math.pi * x)[None, :] * np.sin(math.pi * x)[:, None]
    rng = np.random.default_rng(seed)
    f = f + rng.uniform(-1e-3, 1e-3, size=(n, n))
    b = np.zeros((n + 2, n + 2))
    b[1:-1, 1:-1] = f * h * h
    return so, b


def gaussian_field(ncx, ncy, ell, sigma, seed):
    """Stationary Gaussian random field on the cell centres of the unit square.

    FFT synthesis on a periodic box twice the domain (to suppress wrap-around
    correlation): white noise times the square root of the spectral density of
    the Gaussian covariance exp(-r^2 / (2 ell^2)), scaled to standard deviation
    sigma.
    """
    rng = np.random.default_rng(seed)
    mx, my = 2 * ncx, 2 * ncy
    hx, hy = 1.0 / ncx, 1.0 / ncy
    kx = np.fft.fftfreq(mx, d=hx) * 2 * math.pi
    ky = np.fft.rfftfreq(my, d=hy) * 2 * math.pi
    K2 = kx[:, None] ** 2 + ky[None, :] ** 2
    spec = np.exp(-0.5 * ell * ell * K2)
    noise = rng.standard_normal((mx, my))
    fld = np.fft.irfft2(np.fft.rfft2(noise) * np.sqrt(spec), s=(mx, my))[:ncx, :ncy]
    fld = fld - fld.mean()
    std = fld.std()
    if std > 0:
        fld = fld * (sigma / std)
    return np.ascontiguousarray(fld.T)  # (ncy, ncx)


def inclusions(ncx, ncy, count, contrast, seed, smin=1.0 / 64, smax=1.0 / 8):
    """Multiplicative factor per cell: ``contrast`` inside ``count`` random rectangles."""
    rng = np.random.default_rng(seed)
    fac = np.ones((ncy, ncx))
    xc = (np.arange(ncx) + 0.5) / ncx
    yc = (np.arange(ncy) + 0.5) / ncy
    for _ in range(count):
        w, hgt = rng.uniform(smin, smax, size=2)
        x0, y0 = rng.uniform(0, 1 - w), rng.uniform(0, 1 - hgt)
        mx = (xc >= x0) & (xc < x0 + w)
        my = (yc >= y0) & (yc < y0 + hgt)
        fac[np.ix_(my, mx)] = contrast
    return fac


def hetero_coefficients(n, ell=1.0 / 32, sigma=2.0, n_incl=64, contrast=1e4, aniso=1e-3,
                        seed_field=1, seed_incl=2):
    """(kx, ky) per cell for an (n+1) x (n+1) cell mesh."""
    nc = n + 1
    k = np.exp(gaussian_field(nc, nc, ell, sigma, seed_field))
    if n_incl:
        k = k * inclusions(nc, nc, n_incl, contrast, seed_incl)
    kx = k
    ky = k.copy()
    if aniso is not None and aniso != 1.0:
        yc = (np.arange(nc) + 0.5) / nc
        ky[yc > 0.5, :] *= aniso
    return kx, ky


def hetero_diffusion(n, ell=1.0 / 32, sigma=2.0, n_incl=64, contrast=1e4, aniso=1e-3,
                     seed_field=1, seed_incl=2, seed_rhs=3):
    """9-point heterogeneous diffusion problem on n x n interior nodes."""
    kx, ky = hetero_coefficients(n, ell, sigma, n_incl, contrast, aniso, seed_field, seed_incl)
    so = gallery.fe_hetero(kx, ky)
    h = 1.0 / (n + 1)
    rng = np.random.default_rng(seed_rhs)
    b = np.zeros((n + 2, n + 2))
    b[1:-1, 1:-1] = rng.uniform(0.0, 1.0, size=(n, n)) * h * h
    return so, b


def inverse_problem(n, n_src=8, ell=1.0 / 32, sigma=1.0, seed_theta=8, seed_src=9, seed_obs=10):
    """Inverse-diffusion setup on (n+1)^2 cells: (theta, theta_obs, f).

    theta, theta_obs: log-coefficient Gaussian fields (cells); f: n_src unit point
    sources at seeded interior nodes (ghost-inclusive node array)."""
    nc = n + 1
    theta = gaussian_field(nc, nc, ell, sigma, seed_theta)
    theta_obs = gaussian_field(nc, nc, ell, sigma, seed_obs)
    rng = np.random.default_rng(seed_src)
    f = np.zeros((n + 2, n + 2))
    pts = rng.integers(1, n + 1, size=(n_src, 2))
    for i, j in pts:
        f[j, i] += 1.0
    return theta, theta_obs, f


def fd_cells(n, count=32, seed=11):
    """Seeded cell indices (cj, ci) for finite-difference checks."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, n + 1, size=(count, 2))


def gaussian_field3(nc, ell, sigma, seed):
    """Stationary Gaussian random field on the cell centres of the unit cube,
    nc cells per axis: FFT synthesis on the periodic box of the domain (white
    noise times the square root of the spectral density of the Gaussian
    covariance exp(-r^2 / (2 ell^2))), scaled to standard deviation sigma.
    Returns (nc, nc, nc) indexed (z, y, x)."""
    rng = np.random.default_rng(seed)
    h = 1.0 / nc
    kx = np.fft.fftfreq(nc, d=h) * 2 * math.pi
    kz = np.fft.rfftfreq(nc, d=h) * 2 * math.pi
    K2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    spec = np.sqrt(np.exp(-0.5 * ell * ell * K2))
    noise = rng.standard_normal((nc, nc, nc))
    fld = np.fft.irfftn(np.fft.rfftn(noise) * spec, s=(nc, nc, nc), axes=(0, 1, 2))
    fld -= fld.mean()
    std = fld.std()
    if std > 0:
        fld *= sigma / std
    return np.ascontiguousarray(fld)


def inclusions3(nc, count, contrast, seed, smin=1.0 / 32, smax=1.0 / 8):
    """Multiplicative factor per cell: ``contrast`` inside ``count`` random boxes."""
    rng = np.random.default_rng(seed)
    fac = np.ones((nc, nc, nc))
    c = (np.arange(nc) + 0.5) / nc
    for _ in range(count):
        w = rng.uniform(smin, smax, size=3)
        o = rng.uniform(0, 1 - w)
        mx = (c >= o[0]) & (c < o[0] + w[0])
        my = (c >= o[1]) & (c < o[1] + w[1])
        mz = (c >= o[2]) & (c < o[2] + w[2])
        fac[np.ix_(mz, my, mx)] = contrast
    return fac


def hetero3_coefficients(n, ell=1.0 / 16, sigma=1.5, n_incl=16, contrast=1e3, seed_field=4, seed_incl=5):
    """Cell coefficient k = exp(g) * inclusions on an (n+1)^3 cell mesh, (z, y, x)."""
    nc = n + 1
    k = np.exp(gaussian_field3(nc, ell, sigma, seed_field))
    if n_incl:
        k *= inclusions3(nc, n_incl, contrast, seed_incl)
    return k


def hetero3_rhs(n, seed=6):
    """b = U[-1, 1] h^3 on the n^3 interior nodes (ghost-inclusive array)."""
    h = 1.0 / (n + 1)
    rng = np.random.default_rng(seed)
    b = np.zeros((n + 2, n + 2, n + 2))
    b[1:-1, 1:-1, 1:-1] = rng.uniform(-1.0, 1.0, size=(n, n, n)) * h ** 3
    return b


def batch_sizes(count=512, seed=7):
    """Edge sizes of the batched workload: drawn from {63,127,255,511,1023} with weights 8:4:2:1:1."""
    rng = np.random.default_rng(seed)
    sizes = np.array([63, 127, 255, 511, 1023])
    w = np.array([8, 4, 2, 1, 1], dtype=float)
    return rng.choice(sizes, size=count, p=w / w.sum())
