"""The oracle's project-written FFTW 3.3.10 / GSL 2.7.1 shims (oracle/shim/), which stand in
for the libraries the reference links (neither is in this image), checked against numpy and
scipy on the operations the reference calls: the 3-D complex DFT of both signs
(fftw_plan_dft_3d, field.hpp:321), normalised associated Legendre functions
(gsl_sf_legendre_sphPlm, tools.hpp:59), spherical Bessel functions (gsl_sf_bessel_jl,
bessel.hpp:20), Wigner 3j symbols (gsl_sf_coupling_3j, common.hpp:29) and the natural cubic
spline (gsl_spline with gsl_interp_cspline, bessel.hpp:23-36).  The shims are evaluated by
oracle/_ref/shim_check (oracle/shim_check.cpp, built here with g++ if absent)."""
import math
import os
import subprocess
import tempfile

import numpy as np
import pytest
import scipy.interpolate
import scipy.special

from conftest import ROOT

EXE = os.path.join(ROOT, "oracle", "_ref", "shim_check")


@pytest.fixture(scope="module")
def shim():
    src = os.path.join(ROOT, "oracle", "shim_check.cpp")
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < os.path.getmtime(src):
        p = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "shim"], capture_output=True, text=True)
        assert p.returncode == 0, p.stdout + p.stderr
    tmp = tempfile.mkdtemp(prefix="hg_shim_")

    def run(op, args, data):
        fin, fout = os.path.join(tmp, "in.f64"), os.path.join(tmp, "out.f64")
        np.ascontiguousarray(data, dtype=np.float64).tofile(fin)
        p = subprocess.run([EXE, op, *map(str, args), fin, fout], capture_output=True, text=True, timeout=120)
        assert p.returncode == 0, p.stderr
        return np.fromfile(fout, dtype=np.float64)

    return run


@pytest.mark.parametrize("shape", [(8, 8, 8), (4, 6, 10), (5, 7, 3), (13, 23, 4), (32, 16, 9)])
@pytest.mark.parametrize("sign", [-1, +1])
def test_fft_3d(shim, shape, sign):
    """Radix-2 and mixed / prime lengths (13 and 23 are factors of the reference's survey
    meshes 260 and 460): agreement with numpy.fft to a few units of 1e-16 of the largest
    output."""
    rng = np.random.default_rng(sum(shape) + sign)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    got = shim("fft", (*shape, sign), a.view(np.float64).ravel()).view(np.complex128).reshape(shape)
    want = np.fft.fftn(a) if sign < 0 else np.fft.ifftn(a) * a.size
    err = np.max(np.abs(got - want)) / np.max(np.abs(want))
    assert err < 2e-15, err


def test_legendre_sphplm(shim):
    """sqrt((2l+1)/4pi (l-m)!/(l+m)!) P_l^m(x), Condon-Shortley phase included (scipy's
    lpmv carries it)."""
    rows = []
    for l in range(0, 11):
        for m in range(0, l + 1):
            for x in np.linspace(-1.0, 1.0, 17):
                rows.append((l, m, x))
    rows = np.array(rows)
    got = shim("plm", (), rows.ravel())
    want = np.array([math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(int(l - m)) / math.factorial(int(l + m)))
                     * scipy.special.lpmv(m, l, x) for l, m, x in rows])
    assert np.max(np.abs(got - want)) < 1e-13 * max(1.0, np.max(np.abs(want)))


def test_spherical_bessel(shim):
    """j_l(x) over the three regimes of the shim (series, Miller downward, upward recurrence),
    l = 0..8, x in [0, 200]: absolute agreement with scipy at 1e-14 (|j_l| <= 1)."""
    xs = np.concatenate([[0.0, 1e-8, 1e-3, 0.5, 0.999, 1.0, 1.001], np.linspace(0.01, 20.0, 400),
                         np.linspace(20.0, 200.0, 200)])
    rows = np.array([(l, x) for l in range(0, 9) for x in xs])
    got = shim("jl", (), rows.ravel())
    want = scipy.special.spherical_jn(rows[:, 0].astype(int), rows[:, 1])
    assert np.max(np.abs(got - want)) < 1e-14


def test_wigner_3j(shim):
    """Racah's sum against sympy's exact 3j symbols for every (j1 j2 j3; m1 m2 m3) with
    j <= 4 that the selection rules allow, and zeros where they forbid."""
    from sympy.physics.wigner import wigner_3j
    rows, want = [], []
    for j1 in range(0, 5):
        for j2 in range(0, 5):
            for j3 in range(abs(j1 - j2), j1 + j2 + 1):
                for m1 in range(-j1, j1 + 1):
                    for m2 in range(-j2, j2 + 1):
                        m3 = -m1 - m2
                        if abs(m3) > j3:
                            continue
                        rows.append((2 * j1, 2 * j2, 2 * j3, 2 * m1, 2 * m2, 2 * m3))
                        want.append(float(wigner_3j(j1, j2, j3, m1, m2, m3)))
    rows.append((2, 2, 2, 2, 0, 0))  # m1 + m2 + m3 != 0
    want.append(0.0)
    got = shim("w3j", (), np.array(rows, dtype=np.float64).ravel())
    assert np.max(np.abs(got - np.array(want))) < 1e-14


def test_natural_cubic_spline(shim):
    """The natural spline through unevenly spaced knots, evaluated at the knots and between
    them, against scipy's CubicSpline(bc_type='natural')."""
    rng = np.random.default_rng(7)
    x = np.cumsum(rng.uniform(0.1, 1.0, 60))
    y = np.sin(x) + 0.1 * rng.standard_normal(60)
    q = np.concatenate([x, rng.uniform(x[0], x[-1], 500)])
    got = shim("spline", (len(x),), np.concatenate([x, y, q]))
    want = scipy.interpolate.CubicSpline(x, y, bc_type="natural")(q)
    assert np.max(np.abs(got - want)) < 1e-13
