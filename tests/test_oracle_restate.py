"""The numpy restatement oracle (oracle/restate.py) against the reference's own outputs
(golden fixtures written by the reference's code), and known-answer tests of the schemes
the reference does not have (PCS, interlacing), for which the restatement is the oracle.
CPU only."""
import numpy as np
import pytest

from conftest import load_golden, relerr

from oracle import restate as R


def kbins(arr):
    return R.bins(float(arr[0]), float(arr[1]), int(arr[2]))


@pytest.mark.parametrize("n_mesh", [32, 64])
@pytest.mark.parametrize("assign", ["NGP", "CIC", "TSC"])
def test_restated_pk_matches_reference(n_mesh, assign):
    d = load_golden("box_pk.npz")
    kb = kbins(d["binning"])
    for ell in (0, 2, 4):
        pk, nm, norm = R.pk_box(d["pos"], n_mesh, float(d["boxsize"]), kb, ell, R.SCHEMES[assign])
        assert relerr(norm * pk, d[f"pk_{n_mesh}_{assign}_{ell}"], 1e-12) < 1e-10, ell


@pytest.mark.parametrize("mp", [(0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2)])
def test_restated_bk_matches_reference(mp):
    d = load_golden("box_bk.npz")
    kb = kbins(d["binning"])
    bk, sn, norm = R.bk_box(d["pos"], int(d["n_mesh"]), float(d["boxsize"]), kb, *mp, R.TSC)
    assert relerr(norm * (bk - sn), d["bk_TSC_" + "".join(map(str, mp))], 1e-12) < 1e-10


@pytest.mark.parametrize("assign", ["NGP", "CIC", "TSC"])
def test_restated_flat_index_rule_matches_reference(assign):
    """Particles on cell edges and box faces: the reference's flat-index bleed / drop rule."""
    d = load_golden("box_edges.npz")
    kb = kbins(d["binning"])
    for ell in (0, 2):
        pk, nm, norm = R.pk_box(d["pos"], 16, float(d["boxsize"]), kb, ell, R.SCHEMES[assign])
        assert relerr(norm * pk, d[f"pk_{assign}_{ell}"], 1e-12) < 1e-10
    bk, sn, norm = R.bk_box(d["pos"], 16, float(d["boxsize"]), kb, 0, 0, 0, R.SCHEMES[assign])
    assert relerr(norm * (bk - sn), d[f"bk_{assign}_000"], 1e-12) < 1e-10


def test_alias_sums_match_direct_image_sums():
    """C_p = sum_n W_p^2 and D_p = sum_n (-1)^n W_p^2 over the images k + 2 k_N n."""
    x = np.linspace(-0.49, 0.49, 37)  # k / (2 k_N)
    n = np.arange(-4000, 4001)
    for scheme in (R.NGP, R.CIC, R.TSC, R.PCS):
        p = scheme + 1
        sinc = np.sinc(x[:, None] + n[None, :]) ** (2 * p)
        C = sinc.sum(axis=1)
        D = (sinc * (-1.0) ** (n[None, :] % 2)).sum(axis=1)
        s, c = np.sin(np.pi * x), np.cos(np.pi * x)
        tail = 2e-3 if p == 1 else 1e-9  # NGP's image sum converges as 1/n
        assert np.max(np.abs(R.alias_c(scheme, s) - C)) < tail, scheme
        assert np.max(np.abs(R.alias_d(scheme, c) - D)) < tail, scheme


@pytest.mark.parametrize("assign", ["CIC", "TSC", "PCS"])
def test_interlaced_shot_noise_kat(assign):
    """Known answer: for a Poisson (uniform) catalogue the shot-noise-subtracted, window-
    corrected P_0 of the interlaced field is consistent with zero in every bin (the
    interlaced aliasing sum keeps only even images); for CIC and TSC the plain shot-noise
    function leaves a bias of many sigma near the Nyquist frequency."""
    rng = np.random.default_rng(7)
    L, n, npart = 1000.0, 32, 200000
    pos = rng.uniform(0.0, L, size=(npart, 3))
    kb = R.bins(0.01, 0.09, 9)  # up to 0.9 k_Nyquist
    pk, nm, norm = R.pk_box(pos, n, L, kb, 0, R.SCHEMES[assign], interlace=True)
    shot = L ** 3 / npart
    sigma = shot * np.sqrt(2.0 / nm)  # Gaussian scatter of a binned power, generous
    assert np.all(np.abs(norm * pk.real) < 5.0 * sigma + 1e-3 * shot), (norm * pk.real / shot)
    if assign == "PCS":  # PCS aliasing is too weak for the negative control below
        return
    # the same field with the non-interlaced C(k) is biased at the highest bins
    box = R.Box(n, L, R.SCHEMES[assign], interlace=True)
    d = R.density_spectrum(box, pos)
    plain = R.Box(n, L, R.SCHEMES[assign], interlace=False, periodic=True)
    plain.W, plain.kmag = box.W, box.kmag
    wrong, _ = R.pk_binned(plain, d, d, kb, float(npart), 0, 0)
    assert abs(box.volume / npart ** 2 * wrong.real[-1]) > 5.0 * sigma[-1]


def test_single_particle_ngp_flat_spectrum():
    """Known answer: one particle at a cell centre, NGP, no window correction needed beyond
    W: |delta(k)|^2 is flat, so every bin of the raw binned power equals its analytic value."""
    L, n = 100.0, 16
    pos = np.array([[3.0 * L / n, 5.0 * L / n, 7.0 * L / n]])
    box = R.Box(n, L, R.NGP)
    d = R.density_spectrum(box, pos)
    k0 = d.flat[0]
    other = np.delete(d.ravel(), 0)
    assert np.allclose(np.abs(other), 1.0, rtol=1e-13)  # dV * (1/dV) = 1 per mode
    assert abs(k0) < 1e-12


@pytest.mark.parametrize("assign", ["NGP", "CIC", "TSC"])
def test_restated_outside_box_matches_reference(assign):
    """Particles beyond the box faces and up to three box lengths away: int() truncation
    toward zero (CIC/TSC weights above 1 for negative coordinates) and the flat-index rule."""
    d = load_golden("box_outside.npz")
    kb = kbins(d["binning"])
    for ell in (0, 2):
        pk, nm, norm = R.pk_box(d["pos"], int(d["n_mesh"]), float(d["boxsize"]), kb, ell, R.SCHEMES[assign])
        assert relerr(norm * pk, d[f"pk_{assign}_{ell}"], 1e-12) < 1e-10
    bk, sn, norm = R.bk_box(d["pos"], int(d["n_mesh"]), float(d["boxsize"]), kb, 0, 0, 0, R.SCHEMES[assign])
    assert relerr(norm * (bk - sn), d[f"bk_{assign}_000"], 1e-12) < 1e-10


@pytest.mark.parametrize("assign", ["TSC", "CIC"])
def test_restated_pk_mixed_mesh_matches_reference(assign):
    """A [60, 36, 50] mesh of a [1000, 800, 900] box: lengths that are not powers of two and
    unequal cells (numpy's FFT takes any length, as FFTW does for the reference)."""
    d = load_golden("mixed_meshes.npz")
    kb = kbins(d["box_binning"])
    nm = [int(v) for v in d["box_n_mesh"]]
    bs = [float(v) for v in d["box_boxsize"]]
    for ell in (0, 2):
        pk, nmode, norm = R.pk_box(d["box_pos"], nm, bs, kb, ell, R.SCHEMES[assign])
        assert relerr(norm * pk, d[f"box_pk_{assign}_{ell}"], 1e-12) < 1e-10, ell


def test_restated_bk_unequal_cells_matches_reference():
    """B_202 on a [64, 36, 50] mesh of a [1000, 800, 900] box: the shot noise's per-cell |r|
    with unequal cells (the reference's field.hpp:1040-1050 rvec)."""
    d = load_golden("general_meshes.npz")
    kb = kbins(d["box_binning"])
    nm = [int(v) for v in d["box_n_mesh"]]
    bs = [float(v) for v in d["box_boxsize"]]
    bk, sn, norm = R.bk_box(d["box_pos"], nm, bs, kb, 2, 0, 2, R.TSC)
    assert relerr(norm * (bk - sn), d["box_bk_202"], 1e-12) < 1e-10
