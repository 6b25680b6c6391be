"""TEST INFRASTRUCTURE ONLY: a numpy restatement of the reference's periodic-box
estimators (P_l and B_l), written from src/hitomi_measurement/{field,powerspec,bispec,
tools,bessel}.hpp, plus the schemes the reference does not have (PCS assignment and
interlacing), for which it is the oracle.

It is pinned against the reference itself: tests/test_oracle_restate.py checks it against
the golden fixtures that the reference's own code wrote (tests/golden/box_pk.npz,
box_bk.npz, box_edges.npz) to 1e-10.  Only tests/ and the fixture script import it.

Every function states the reference lines it follows.  Conventions: FFT_- = numpy.fft.fftn
(FFTW_FORWARD), FFT_+ = N * numpy.fft.ifftn (FFTW_BACKWARD, unnormalised); arrays are
[x][y][z] row-major like the reference's `coord = (i*Ny + j)*Nz + k`.
"""
from __future__ import annotations

import numpy as np
from scipy.interpolate import CubicSpline
from scipy.special import sph_harm_y, spherical_jn

NGP, CIC, TSC, PCS = 0, 1, 2, 3
SCHEMES = {"NGP": NGP, "CIC": CIC, "TSC": TSC, "PCS": PCS}


def bins(vmin: float, vmax: float, n: int) -> np.ndarray:
    """tools.hpp:118-134: vmin + d * i with d = (vmax - vmin) / (n - 1)."""
    d = (vmax - vmin) / float(n - 1)
    return np.array([vmin + d * float(i) for i in range(n)])


def wrap(i: np.ndarray, n: int) -> np.ndarray:
    """Mode / offset index of array index i: i for i < n/2, i - n otherwise (field.hpp:362-364)."""
    return np.where(i < n // 2, i, i - n)


def ylm_reduced(l: int, m: int, x, y, z) -> np.ndarray:
    """Yhat_lm(v) = conj(Y_lm(v_hat)) sqrt(4 pi / (2l+1)); 1 for l = m = 0, 0 for |v| < 1e-15
    (tools.hpp:12-68).  Y_lm with the Condon-Shortley phase (scipy's sph_harm_y)."""
    x, y, z = (np.asarray(v, dtype=np.float64) for v in (x, y, z))
    if l == 0 and m == 0:
        return np.ones(np.broadcast(x, y, z).shape, dtype=np.complex128)
    r = np.sqrt(x * x + y * y + z * z)
    ok = np.abs(r) >= 1e-15
    rs = np.where(ok, r, 1.0)
    theta = np.arccos(np.clip(z / rs, -1.0, 1.0))
    phi = np.arctan2(y, x)
    out = np.conj(sph_harm_y(l, m, theta, phi)) * np.sqrt(4.0 * np.pi / (2 * l + 1))
    return np.where(ok, out, 0.0)


# ---------------------------------------------------------------- assignment
def _axis_stencil(xp: np.ndarray, scheme: int):
    """Anchor index and per-point weights per axis: field.hpp:80-90 (NGP), 117-129 (CIC),
    158-172 (TSC); PCS (not in the reference) is the cubic B-spline on floor(xp) - 1 .. + 2."""
    if scheme == NGP:
        i = (xp + 0.5).astype(np.int64)
        return i, [np.ones_like(xp)]
    if scheme == CIC:
        i = xp.astype(np.int64)
        d = xp - i
        return i, [1.0 - d, d]
    if scheme == TSC:
        i = (xp + 0.5).astype(np.int64)
        d = xp - i
        return i - 1, [0.5 * (0.5 - d) * (0.5 - d), 0.75 - d * d, 0.5 * (0.5 + d) * (0.5 + d)]
    i = np.floor(xp).astype(np.int64)
    t = xp - i
    u = 1.0 - t
    return i - 1, [u * u * u / 6.0, (4.0 - 6.0 * t * t + 3.0 * t * t * t) / 6.0,
                   (1.0 + 3.0 * t + 3.0 * t * t - 3.0 * t * t * t) / 6.0, t * t * t / 6.0]


def assign(pos, n_mesh, boxsize, scheme: int, periodic: bool = False, shift: float = 0.0, weights=None,
           factor: float | None = None) -> np.ndarray:
    """rho(x) = sum_p w_p factor prod_axis W_axis with factor = 1/dV (field.hpp:67-184).
    periodic = False keeps the reference's flat-index rule (only 0 <= coord < N is tested,
    field.hpp:92-96); periodic = True wraps every axis (PCS / interlacing).  shift (in cells)
    is added to the scaled position (the interlaced copy uses 0.5)."""
    n = np.broadcast_to(np.asarray(n_mesh), (3,)).astype(np.int64)
    L = np.broadcast_to(np.asarray(boxsize, dtype=np.float64), (3,))
    pos = np.asarray(pos, dtype=np.float64)
    npart = pos.shape[0]
    vol = float(L[0] * L[1] * L[2])
    if factor is None:
        factor = 1.0 / (vol / float(n[0] * n[1] * n[2]))
    w = np.ones(npart, dtype=np.complex128) if weights is None else np.asarray(weights, dtype=np.complex128)
    anc, wts = [], []
    for a in range(3):
        xp = pos[:, a] * float(n[a]) / L[a]
        if shift != 0.0:
            xp = xp + shift
        i0, ws = _axis_stencil(xp, scheme)
        anc.append(i0)
        wts.append(ws)
    ntot = int(n[0] * n[1] * n[2])
    rho = np.zeros(ntot, dtype=np.complex128)
    W = len(wts[0])
    for a in range(W):
        for b in range(W):
            for c in range(W):
                ix, iy, iz = anc[0] + a, anc[1] + b, anc[2] + c
                if periodic:
                    coord = ((ix % n[0]) * n[1] + (iy % n[1])) * n[2] + (iz % n[2])
                    ok = np.ones(npart, dtype=bool)
                else:
                    coord = (ix * n[1] + iy) * n[2] + iz
                    ok = (coord >= 0) & (coord < ntot)
                val = w * factor * wts[0][a] * wts[1][b] * wts[2][c]
                np.add.at(rho, coord[ok], val[ok])
    return rho.reshape(tuple(n))


# ---------------------------------------------------------------- Fourier-space weights
def axis_tables(n: int, L: float, exact: bool):
    """Per-axis window / shot-noise factors.  The reference's index is
    (int)(k / dk + 1e-5) -- n + 1 for negative modes (field.hpp:664-675, 1261-1272);
    exact = True uses the mode index (PCS, interlacing).  Returns (sinc, sin, cos) of
    pi w / n."""
    dk = 2.0 * np.pi / L
    i = np.arange(n)
    kv = wrap(i, n).astype(np.float64) * dk
    w = wrap(i, n) if exact else np.trunc(kv / dk + 1e-5).astype(np.int64)
    x = np.pi * w.astype(np.float64) / float(n)
    sinc = np.where(w == 0, 1.0, np.sin(x) / np.where(w == 0, 1.0, x))
    return sinc, np.where(w == 0, 0.0, np.sin(x)), np.where(w == 0, 1.0, np.cos(x))


def alias_c(scheme: int, s):
    """sum over images of W^2 per axis (field.hpp:1252-1310; PCS from the same sum)."""
    s2 = s * s
    if scheme == NGP:
        return np.ones_like(s)
    if scheme == CIC:
        return 1.0 - (2.0 / 3.0) * s2
    if scheme == TSC:
        return 1.0 - s2 + 2.0 * (s2 * s2) / 15.0
    return 1.0 - (4.0 / 3.0) * s2 + (2.0 / 5.0) * s2 * s2 - (4.0 / 315.0) * s2 * s2 * s2


def alias_d(scheme: int, c):
    """sum over images of (-1)^n W^2 per axis (closed form of the alternating sinc^2p sum)."""
    c2 = c * c
    if scheme == NGP:
        return c
    if scheme == CIC:
        return c * (c2 + 5.0) / 6.0
    if scheme == TSC:
        return c * (c2 * c2 + 58.0 * c2 + 61.0) / 120.0
    return c * (c2 * c2 * c2 + 543.0 * c2 * c2 + 3111.0 * c2 + 1385.0) / 5040.0


class Box:
    """Grid geometry and the per-mode arrays the estimators use."""

    def __init__(self, n_mesh, boxsize, scheme: int, interlace: bool = False, periodic: bool = False):
        self.n = np.broadcast_to(np.asarray(n_mesh), (3,)).astype(np.int64)
        self.L = np.broadcast_to(np.asarray(boxsize, dtype=np.float64), (3,))
        self.scheme = scheme
        self.interlace = interlace
        self.periodic = periodic or interlace or scheme == PCS
        self.exact = interlace or scheme == PCS
        self.ntot = int(self.n.prod())
        self.volume = float(self.L[0] * self.L[1] * self.L[2])
        self.dV = self.volume / float(self.ntot)
        dk = 2.0 * np.pi / self.L
        idx = [np.arange(int(m)) for m in self.n]
        self.kv = [wrap(idx[a], int(self.n[a])).astype(np.float64) * dk[a] for a in range(3)]
        dr = self.L / self.n.astype(np.float64)
        self.rv = [wrap(idx[a], int(self.n[a])).astype(np.float64) * dr[a] for a in range(3)]
        KX, KY, KZ = np.meshgrid(*self.kv, indexing="ij")
        self.k = (KX, KY, KZ)
        self.kmag = np.sqrt(KX * KX + KY * KY + KZ * KZ)  # field.hpp:366, same operation order
        RX, RY, RZ = np.meshgrid(*self.rv, indexing="ij")
        self.r = (RX, RY, RZ)
        self.rmag = np.sqrt(RX * RX + RY * RY + RZ * RZ)
        tabs = [axis_tables(int(self.n[a]), float(self.L[a]), self.exact) for a in range(3)]
        sx, sy, sz = np.meshgrid(tabs[0][0], tabs[1][0], tabs[2][0], indexing="ij")
        ret = sx * sy * sz
        p = scheme + 1
        Wk = ret.copy()
        for _ in range(1, p):
            Wk = Wk * ret
        self.W = Wk
        ax = [(alias_c(scheme, tabs[a][1]), alias_d(scheme, tabs[a][2])) for a in range(3)]
        cx, cy, cz = np.meshgrid(ax[0][0], ax[1][0], ax[2][0], indexing="ij")
        C = cx * cy * cz
        if interlace:
            dx, dy, dz = np.meshgrid(ax[0][1], ax[1][1], ax[2][1], indexing="ij")
            C = 0.5 * (C + dx * dy * dz)
        self.C = C

    def ylm_k(self, l, m):
        return ylm_reduced(l, m, *self.k)

    def ylm_x(self, l, m):
        return ylm_reduced(l, m, *self.r)


def density_spectrum(box: Box, pos) -> np.ndarray:
    """FFT_-[dV (rho - N/V)] (field.hpp:505-525, 310-325); with interlacing, the average of
    the plain and the half-cell shifted assignments, (F_0 + e^{i pi (nx/Nx+ny/Ny+nz/Nz)} F_s)/2,
    formed on the half spectrum (nz >= 0) and extended by Hermitian symmetry."""
    npart = pos.shape[0]
    nbar = float(npart) / box.volume
    rho = assign(pos, box.n, box.L, box.scheme, box.periodic).real
    if not box.interlace:
        return np.fft.fftn(box.dV * (rho - nbar))
    rho_s = assign(pos, box.n, box.L, box.scheme, box.periodic, shift=0.5).real
    h0 = np.fft.rfftn(box.dV * (rho - nbar))
    h1 = np.fft.rfftn(box.dV * (rho_s - nbar))
    n0, n1, n2 = (int(v) for v in box.n)
    qx = wrap(np.arange(n0), n0) / n0
    qy = wrap(np.arange(n1), n1) / n1
    qz = np.arange(n2 // 2 + 1) / n2
    q = qx[:, None, None] + qy[None, :, None] + qz[None, None, :]
    h = 0.5 * (h0 + np.exp(1j * np.pi * q) * h1)
    return hermitian_full(h, n2)


def hermitian_full(h: np.ndarray, n2: int) -> np.ndarray:
    n0, n1, hz = h.shape
    full = np.empty((n0, n1, n2), dtype=np.complex128)
    full[:, :, :hz] = h
    ix = (-np.arange(n0)) % n0
    iy = (-np.arange(n1)) % n1
    for iz in range(hz, n2):
        full[:, :, iz] = np.conj(h[ix][:, iy, n2 - iz])
    return full


# ---------------------------------------------------------------- power spectrum
def pk_binned(box: Box, f1, f2, kbin, S, l, m):
    """TwoPointStatisticsClass::calcPowerSpectrum (field.hpp:765-852): fine histogram
    int(|k|/1e-4 + 0.5) < 1e5 of (f1 conj f2 - S C(k)) / W^2 Yhat_lm(k), then coarse bins
    (lower, upper] on i * 1e-4 with lower = kbin - dk/2 (0 below dk/2), upper = kbin + dk/2.
    Returns (pk averaged per bin, n_mode)."""
    dkb = kbin[1] - kbin[0]
    kidx = (box.kmag / 0.0001 + 0.5).astype(np.int64).ravel()
    ok = kidx < 100000
    pk2 = (f1 * np.conj(f2) - S * box.C) / box.W ** 2 * box.ylm_k(l, m)
    fine = np.zeros(100000, dtype=np.complex128)
    cnt = np.zeros(100000, dtype=np.int64)
    np.add.at(fine, kidx[ok], pk2.ravel()[ok])
    np.add.at(cnt, kidx[ok], 1)
    kt = np.arange(100000) * 0.0001
    pk = np.zeros(len(kbin), dtype=np.complex128)
    nm = np.zeros(len(kbin), dtype=np.int64)
    for j, kc in enumerate(kbin):
        lower = (kc - dkb * 0.5) if kc > dkb * 0.5 else 0.0
        upper = kc + dkb * 0.5
        sel = (kt > lower) & (kt <= upper)
        pk[j] = fine[sel].sum()
        nm[j] = cnt[sel].sum()
    return np.where(nm != 0, pk / np.maximum(nm, 1), 0.0), nm


def pk_box(pos, n_mesh, boxsize, kbin, ell: int, scheme: int, interlace: bool = False, periodic: bool = False):
    """calcPowerSpectrumForBOX (powerspec.hpp:273-332): (2l+1) P_hat with Y_l0, shot noise N,
    norm V / N^2.  Returns (pk_save, n_mode, norm)."""
    box = Box(n_mesh, boxsize, scheme, interlace, periodic)
    d = density_spectrum(box, pos)
    npart = float(pos.shape[0])
    pk, nm = pk_binned(box, d, d, kbin, npart, ell, 0)
    return (2 * ell + 1) * pk, nm, box.volume / npart / npart


# ---------------------------------------------------------------- bispectrum
class Bessel:
    """SphericalBesselClass (bessel.hpp:10-37): natural cubic spline of j_l through 10^6
    knots on [0, 10^4]."""

    def __init__(self, ell: int):
        n = 1000000
        dx = (10000.0 - 0.0) / float(n - 1)
        x = 0.0 + dx * np.arange(n, dtype=np.float64)
        self.s = CubicSpline(x, spherical_jn(ell, x), bc_type="natural")

    def __call__(self, x):
        return self.s(x)


def wigner3j(j1, j2, j3, m1, m2, m3) -> float:
    """Racah's formula (the value gsl_sf_coupling_3j returns, common.hpp:29)."""
    from math import factorial, sqrt
    if m1 + m2 + m3 != 0 or j3 < abs(j1 - j2) or j3 > j1 + j2 or abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    f = factorial
    tri = f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3) / f(j1 + j2 + j3 + 1)
    pre = sqrt(tri * f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3))
    s = 0.0
    for t in range(0, j1 + j2 + j3 + 2):
        den = [t, j3 - j2 + t + m1, j3 - j1 + t - m2, j1 + j2 - j3 - t, j1 - t - m1, j2 - t + m2]
        if min(den) < 0:
            continue
        v = 1.0
        for q in den:
            v *= f(q)
        s += (-1) ** t / v
    return (-1) ** (j1 - j2 - m3) * pre * s


def combos(l1, l2, L):
    """(m1, m2) with M = 0 and |w| >= 1e-10, w = (2L+1)(2l1+1)(2l2+1) w3j(l1 l2 L;000) w3j(l1 l2 L;m1 m2 0)
    (bispec.hpp:1129-1136)."""
    out = []
    for m1 in range(-l1, l1 + 1):
        for m2 in range(-l2, l2 + 1):
            w = wigner3j(l1, l2, L, 0, 0, 0) * wigner3j(l1, l2, L, m1, m2, 0)
            w *= float(2 * L + 1) * float(2 * l1 + 1) * float(2 * l2 + 1)
            if abs(w) >= 1.0e-10:
                out.append((m1, m2, w))
    return out


def bk_box(pos, n_mesh, boxsize, kbin, l1: int, l2: int, L: int, scheme: int, interlace: bool = False,
           periodic: bool = False):
    """calcBiSpectrumForBOX (bispec.hpp:877-1203) for every k1 row at once.
    Returns (bk_save [n_kbin][n_kbin], sn_save [n_kbin][n_kbin], norm)."""
    box = Box(n_mesh, boxsize, scheme, interlace, periodic)
    d = density_spectrum(box, pos)
    npart = float(pos.shape[0])
    nk = len(kbin)
    dk_in = kbin[1] - kbin[0]
    ntot = box.ntot
    # FFT_-[dV rho] differs from d only at k = 0, by sum_c nbar dV = N (field.hpp:527-560)
    nd = d.copy()
    nd.flat[0] = d.flat[0] + npart
    # G = FFT_+[d / W] / V (field.hpp:326-344 after the window correction)
    G = np.fft.ifftn(d / box.W) * ntot / box.volume
    shells = []
    for kc in kbin:
        lower = (kc - dk_in * 0.5) if kc > dk_in * 0.5 else 0.0
        upper = kc + dk_in * 0.5
        shells.append((box.kmag > lower) & (box.kmag <= upper))
    bk = np.zeros((nk, nk), dtype=np.complex128)
    sn = np.zeros((nk, nk), dtype=np.complex128)
    cmb = combos(l1, l2, L)
    # shell fields (field.hpp:346-401): FFT_+[S_i Yhat d / W] / n_mode_i
    def fields(l, m):
        y = box.ylm_k(l, m)
        return [np.fft.ifftn(np.where(s, y * d / box.W, 0.0)) * ntot / float(s.sum()) for s in shells]
    for m1, m2, w in cmb:
        F1 = fields(l1, m1)
        F2 = F1 if (l1, m1) == (l2, m2) else fields(l2, m2)
        for i1 in range(nk):
            for i2 in range(nk):
                bk[i1, i2] += w * (box.dV * np.sum(F1[i1] * F2[i2] * G))
    # shot noise (bispec.hpp:909-1078)
    j1s, j2s = Bessel(l1), Bessel(l2)
    for m1, m2, w in cmb:
        if l1 == 0 and l2 == 0:
            sn += w * npart
        if l2 == 0:
            p, _ = pk_binned(box, d, nd, kbin, npart, l1, m1)
            sn += w * p[:, None]  # the k1 row's value on every k2
        if l1 == 0:
            p, _ = pk_binned(box, d, nd, kbin, npart, l2, m2)
            sn += w * p[None, :]
        # xi = FFT_+[(d conj N - N C) / W^2 / V] (field.hpp:1116-1160)
        xi = np.fft.ifftn((d * np.conj(nd) - npart * box.C) / box.W ** 2 / box.volume) * ntot
        yy = box.ylm_x(l1, m1) * box.ylm_x(l2, m2) * xi
        fac = box.volume / float(ntot)
        for i1 in range(nk):
            a = j1s(kbin[i1] * box.rmag) * yy
            for i2 in range(nk):
                s_ = np.sum(j2s(kbin[i2] * box.rmag) * a)
                sn[i1, i2] += w * (s_ * (1j ** (l1 + l2)) * fac)
    norm = box.volume / npart / npart * (box.volume / npart)
    return bk, sn, norm
