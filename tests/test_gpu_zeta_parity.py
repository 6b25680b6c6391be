"""GPU parity of the periodic-box 3PCF multipoles zeta_{l1 l2 L}(r1, r2) against the
reference (golden fixtures written by calcThreePointCorrelationFunctionForBOX,
bispec.hpp:1205-1424, through tests/golden/make_golden.py).

The fixtures hold the reference's file values norm * Re(zeta - sn) for every r1 row.
Tolerances as for P and B: FP64 1e-10 relative per bin; FP32 1e-4 relative to
max(|bin|, 1e-3 max|bins|)."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}
MULTIPOLES = ((0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2), (1, 1, 2))


def ctx(n_mesh, boxsize, b, assign, form):
    from hitomi_b200.api import Context
    return Context(n_mesh, boxsize, b, assign, form)


def file_value(z, sn, norm):
    return norm * (z - sn).real


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_zeta_box_all_multipoles(form):
    d = load_golden("box_zeta.npz")
    b = binning_from(d["binning"])
    with ctx(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", form) as c:
        c.set_particles(0, d["pos"])
        for mp in MULTIPOLES:
            z, sn, norm = c.zeta_box(*mp)
            ref = d["zeta_TSC_" + "".join(map(str, mp))]
            assert relerr(file_value(z, sn, norm), ref, FLOOR[form]) < TOL[form], mp


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign", ["NGP", "CIC"])
def test_zeta_box_other_assignments(form, assign):
    d = load_golden("box_zeta.npz")
    b = binning_from(d["binning"])
    with ctx(int(d["n_mesh"]), float(d["boxsize"]), b, assign, form) as c:
        c.set_particles(0, d["pos"])
        z, sn, norm = c.zeta_box(0, 0, 0)
        assert relerr(file_value(z, sn, norm), d[f"zeta_{assign}_000"], FLOOR[form]) < TOL[form]


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_zeta_edges_and_wide_bins(form):
    """Boundary-stress catalogue; r bins from below one cell to past half the box."""
    d = load_golden("box_zeta.npz")
    b = binning_from(d["edge_binning"])
    with ctx(16, 400.0, b, "TSC", form) as c:
        c.set_particles(0, d["edge_pos"])
        for mp in ((0, 0, 0), (1, 1, 0)):
            z, sn, norm = c.zeta_box(*mp)
            ref = d["edge_zeta_TSC_" + "".join(map(str, mp))]
            assert relerr(file_value(z, sn, norm), ref, FLOOR[form]) < TOL[form], mp


def test_zeta_single_row_and_shot_noise_diagonal():
    """ith_rbin >= 0 gives that row of the all-rows matrix; shot noise only at r1 = r2."""
    d = load_golden("box_zeta.npz")
    b = binning_from(d["binning"])
    with ctx(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", "fp64") as c:
        c.set_particles(0, d["pos"])
        z_all, sn_all, norm = c.zeta_box(1, 1, 0)
        off = sn_all - np.diag(np.diag(sn_all))
        assert np.all(off == 0)
        for ith in (0, 3, b.n_rbin - 1):
            z, sn, norm1 = c.zeta_box(1, 1, 0, ith)
            assert norm1 == norm
            np.testing.assert_allclose(z[0], z_all[ith], rtol=1e-12, atol=1e-12 * np.abs(z_all).max())
            np.testing.assert_array_equal(sn[0], sn_all[ith])
            ref = d["zeta_TSC_110"][ith]
            assert relerr(file_value(z[0], sn[0], norm1), ref, 1e-12) < 1e-10


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_zeta_box_multi_matches_single(form):
    d = load_golden("box_zeta.npz")
    b = binning_from(d["binning"])
    with ctx(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", form) as c:
        c.set_particles(0, d["pos"])
        zm, snm, norm = c.zeta_box_multi(MULTIPOLES)
        for q, mp in enumerate(MULTIPOLES):
            ref = d["zeta_TSC_" + "".join(map(str, mp))]
            assert relerr(file_value(zm[q], snm[q], norm), ref, FLOOR[form]) < TOL[form], mp


def test_zeta_after_bispectrum_on_same_context():
    """B and zeta share the density transform and shot-noise histograms of one catalogue."""
    d = load_golden("box_zeta.npz")
    b = binning_from(d["binning"])
    with ctx(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", "fp64") as c:
        c.set_particles(0, d["pos"])
        c.bk_box(2, 0, 2)
        z, sn, norm = c.zeta_box(2, 0, 2)
        assert relerr(file_value(z, sn, norm), d["zeta_TSC_202"], 1e-12) < 1e-10


def test_zeta_rejects_bad_rows():
    """(Non-cubic meshes run: tests/test_gpu_general_meshes.py.)"""
    from hitomi_b200.api import Binning, Context, HitomiError
    b = Binning(0.02, 0.1, 5, 20.0, 140.0, 7)
    pos = np.random.default_rng(3).uniform(0, 400.0, size=(1000, 3))
    with Context(16, 400.0, b, "TSC", "fp64") as c:
        c.set_particles(0, pos)
        with pytest.raises(HitomiError, match="ith_rbin"):
            c.zeta_box(0, 0, 0, 7)
        with pytest.raises(HitomiError, match="not allowed"):
            c.zeta_box(1, 0, 0)


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_zeta_box_odd_multipoles(form):
    """l1 + l2 odd: shot-noise weights odd in cos(theta), the Nyquist plane z = -L/2 included."""
    d = load_golden("box_odd.npz")
    b = binning_from(d["zeta_binning"])
    with ctx(int(d["n_mesh"]), float(d["zeta_boxsize"]), b, "TSC", form) as c:
        c.set_particles(0, d["zeta_pos"])
        for mp in ((1, 0, 1), (2, 1, 1)):
            z, sn, norm = c.zeta_box(*mp)
            ref = d["zeta_TSC_" + "".join(map(str, mp))]
            assert relerr(file_value(z, sn, norm), ref, FLOOR[form]) < TOL[form], mp
