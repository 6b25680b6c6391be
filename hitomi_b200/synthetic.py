"""Seeded synthetic catalogues with the shapes of the workloads the estimators run on.

No survey or simulation data ships with this repository; these generators stand in for
them with the sizes and value distributions of the configurations the reference is run
with (periodic N-body boxes, BOSS-like survey shells, many-mock covariance runs).

  uniform_box        positions uniform in [0, L)^3                        (float64)
  lognormal_box      Gaussian field with P(k) = A (k/0.1)^n on a grid, lognormal
                     transform, Poisson sampling, Zel'dovich RSD shift along z, wrapped
  survey_shell       data + randoms in a spherical shell r in [rmin, rmax] cut to a
                     square patch of the sky, Gaussian n(r), FKP weights 1/(1 + n P0)
"""
from __future__ import annotations

import numpy as np


def uniform_box(n: int, boxsize: float = 1000.0, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, boxsize, size=(n, 3))


def _kgrid(ng: int, boxsize: float):
    k1 = 2.0 * np.pi * np.fft.fftfreq(ng, d=boxsize / ng)
    kz1 = 2.0 * np.pi * np.fft.rfftfreq(ng, d=boxsize / ng)
    kx = k1[:, None, None]
    ky = k1[None, :, None]
    kz = kz1[None, None, :]
    return kx, ky, kz


def lognormal_box(n_target: float, boxsize: float = 1000.0, ngrid: int = 256, amp: float = 2.0e4,
                  slope: float = -1.5, f_growth: float = 0.7, seed: int = 2, exact_n: int | None = None) -> np.ndarray:
    """Clustered periodic catalogue.

    delta_G has power spectrum amp (k/0.1)^slope (Mpc/h)^3 on an ngrid^3 mesh of side
    boxsize; the density is n_bar (1 + delta_LN) with delta_LN = exp(delta_G - s^2/2) - 1;
    particle counts per cell are Poisson, positions uniform inside the cell; each particle
    is shifted along z by f_growth * Psi_z (Zel'dovich displacement of delta_G at its cell)
    and wrapped into [0, boxsize).  exact_n, if given, trims or tops up (uniformly) to
    exactly that many particles.
    """
    rng = np.random.default_rng(seed)
    ng = int(ngrid)
    kx, ky, kz = _kgrid(ng, boxsize)
    k2 = kx * kx + ky * ky + kz * kz
    kk = np.sqrt(k2)
    pk = np.zeros_like(kk)
    nz = kk > 0
    pk[nz] = amp * (kk[nz] / 0.1) ** slope
    vol = boxsize ** 3
    # white noise with unit variance per cell -> field with the target power
    white = rng.standard_normal((ng, ng, ng))
    wk = np.fft.rfftn(white)
    dk = wk * np.sqrt(pk * ng ** 3 / vol)
    delta_g = np.fft.irfftn(dk, s=(ng, ng, ng), axes=(0, 1, 2))
    sig2 = float(np.var(delta_g))
    delta_ln = np.exp(delta_g - 0.5 * sig2) - 1.0
    cell = boxsize / ng
    nbar = n_target / vol
    lam = nbar * cell ** 3 * (1.0 + delta_ln)
    counts = rng.poisson(lam.ravel())
    n = int(counts.sum())
    idx = np.repeat(np.arange(ng ** 3, dtype=np.int64), counts)
    ix = idx // (ng * ng)
    iy = (idx // ng) % ng
    iz = idx % ng
    pos = np.empty((n, 3))
    pos[:, 0] = (ix + rng.random(n)) * cell
    pos[:, 1] = (iy + rng.random(n)) * cell
    pos[:, 2] = (iz + rng.random(n)) * cell
    # Zel'dovich displacement Psi(k) = i k / k^2 delta_G(k), z component only
    with np.errstate(divide="ignore", invalid="ignore"):
        psi_k = np.where(k2 > 0, 1j * kz / k2, 0.0) * dk
    psi_z = np.fft.irfftn(psi_k, s=(ng, ng, ng), axes=(0, 1, 2)).ravel()
    pos[:, 2] += f_growth * psi_z[idx]
    pos %= boxsize
    pos[pos >= boxsize] -= boxsize  # guard the round-up of x % L == L
    if exact_n is not None:
        if n >= exact_n:
            sel = rng.permutation(n)[:exact_n]
            pos = pos[np.sort(sel)]
        else:
            extra = rng.uniform(0.0, boxsize, size=(exact_n - n, 3))
            pos = np.concatenate([pos, extra])
    return np.ascontiguousarray(pos)


def survey_shell(n_data: int, n_rand: int, rmin: float = 1000.0, rmax: float = 1800.0, rmean: float = 1400.0,
                 rsig: float = 200.0, npeak: float = 3.0e-4, cap_deg: float = 60.0, p0: float = 1.0e4,
                 seed: int = 3):
    """Survey-like data and randoms as (n, 4) arrays of x y z w (observer at the origin).

    Directions are uniform on the sphere inside the patch |lon| <= cap/2, |lat| <= cap/2
    around the +x axis; radii follow r^2 n(r) with n(r) = npeak exp(-(r-rmean)^2/2 rsig^2)
    on [rmin, rmax]; weights are FKP, w = 1 / (1 + n(r) p0).
    """
    rng = np.random.default_rng(seed)
    half = np.deg2rad(cap_deg / 2.0)

    def draw(n):
        lon = rng.uniform(-half, half, n)
        lat = np.arcsin(rng.uniform(-np.sin(half), np.sin(half), n))
        # rejection sampling of r with density r^2 n(r)
        rs = np.empty(0)
        fmax = rmax ** 2
        while rs.size < n:
            m = 2 * (n - rs.size) + 16
            r = rng.uniform(rmin, rmax, m)
            acc = rng.random(m) < (r * r / fmax) * np.exp(-0.5 * ((r - rmean) / rsig) ** 2)
            rs = np.concatenate([rs, r[acc]])
        r = rs[:n]
        x = r * np.cos(lat) * np.cos(lon)
        y = r * np.cos(lat) * np.sin(lon)
        z = r * np.sin(lat)
        nr = npeak * np.exp(-0.5 * ((r - rmean) / rsig) ** 2)
        w = 1.0 / (1.0 + nr * p0)
        return np.ascontiguousarray(np.stack([x, y, z, w], axis=1))

    return draw(n_data), draw(n_rand)
