"""GPU parity of the two-point correlation function multipoles and the window functions
against the reference (golden fixtures written by calcTwoPointCorrelationFunctionForBOX,
powerspec.hpp:334-393; calcTwoPointCorrelationFunction, powerspec.hpp:93-180;
calcTwoPointWindowCorrelationFunction, powerspec.hpp:182-270; and
calcThreePointWindowCorrelationFunction, bispec.hpp:617-874, through
tests/golden/make_golden.py --xi).  The files hold norm * Re(xi_save) and
norm * Re(zeta_save - sn_save).  Tolerances as the other parity tests: FP64 1e-10 relative
per bin; FP32 1e-4 (3e-4 for the sparse survey 3PCF catalogue) relative to
max(|bin|, 1e-3 max|bins|)."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign,ells", [("TSC", (0, 2, 4)), ("CIC", (0, 2)), ("NGP", (0, 2))])
def test_xi_box(form, assign, ells):
    from hitomi_b200.api import Context
    d = load_golden("xi_window.npz")
    b = binning_from(d["box_binning"])
    with Context(int(d["box_n_mesh"]), float(d["box_boxsize"]), b, assign, form) as c:
        c.set_particles(0, d["box_pos"])
        for ell in ells:
            xi, nmode, norm = c.xi_box(ell)
            assert relerr(norm * xi.real, d[f"box_xi_{assign}_{ell}"], FLOOR[form]) < TOL[form], ell
            # the first bin (0, 8] Mpc/h holds no cell of this 15.6 Mpc/h mesh: xi = 0 there
            assert nmode[0] == 0 and np.all(nmode[1:] > 0)


def test_xi_box_odd_multipole_is_imaginary():
    """Odd l in the box: xi(-x) = conj xi(x) and L_l(mu) is odd, so the multipole is purely
    imaginary and the real part the reference prints is rounding noise on both sides."""
    from hitomi_b200.api import Context
    d = load_golden("xi_window.npz")
    b = binning_from(d["box_binning"])
    with Context(int(d["box_n_mesh"]), float(d["box_boxsize"]), b, "TSC", "fp64") as c:
        c.set_particles(0, d["box_pos"])
        xi, _, norm = c.xi_box(1)
    scale = float(np.max(np.abs(norm * xi.imag)))
    assert scale > 0.0
    assert np.max(np.abs(norm * xi.real)) < 1e-12 * scale
    assert np.max(np.abs(d["box_xi_TSC_1"])) < 1e-12 * scale


def test_xi_box_after_bispectrum_shares_nothing_stale():
    """The box correlation field of the bispectrum shot noise differs from the 2PCF's at
    k = 0 (dn against the density, not itself): mixing the calls must not reuse it."""
    from hitomi_b200.api import Context
    d = load_golden("xi_window.npz")
    b = binning_from(d["box_binning"])
    with Context(int(d["box_n_mesh"]), float(d["box_boxsize"]), b, "TSC", "fp64") as c:
        c.set_particles(0, d["box_pos"])
        c.bk_box(0, 0, 0)
        xi, _, norm = c.xi_box(0)
        assert relerr(norm * xi.real, d["box_xi_TSC_0"]) < 1e-10
        c.bk_box(2, 0, 2)
        xi, _, norm = c.xi_box(2)
        assert relerr(norm * xi.real, d["box_xi_TSC_2"]) < 1e-10


def survey_records(d, prefix):
    from hitomi_b200 import survey
    nm, bs = int(d[f"{prefix}_n_mesh"]), float(d[f"{prefix}_boxsize"])
    return survey.prepare(d[f"{prefix}_data"], d[f"{prefix}_rand"], nm, bs)


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_xi_survey(form):
    from hitomi_b200.api import Context
    d = load_golden("xi_window.npz")
    b = binning_from(d["sv_binning"])
    D, R = survey_records(d, "sv")
    with Context(int(d["sv_n_mesh"]), float(d["sv_boxsize"]), b, "TSC", form) as c:
        c.set_survey(D, R)
        alpha, vs, *_ = c.survey_scalars()
        for ell in (0, 1, 2):
            xi, _, norm = c.xi_survey(ell, alpha, vs)
            assert relerr(norm * xi.real, d[f"sv_xi_{ell}"], FLOOR[form]) < TOL[form], ell


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("with_data", [False, True])
def test_xi_window(form, with_data):
    """The window function needs the randoms only; with the data also set it ignores them."""
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    d = load_golden("xi_window.npz")
    b = binning_from(d["sv_binning"])
    D, R = survey_records(d, "sv")
    vs = float(d["sv_scalars_vsurvey"])
    with Context(int(d["sv_n_mesh"]), float(d["sv_boxsize"]), b, "TSC", form) as c:
        if with_data:
            c.set_survey(D, R)
        else:
            c.set_particles(1, R, pos_off=survey.POS_OFF, los_off=survey.LOS_OFF, w_off=survey.W_OFF)
        for ell in (0, 1, 2):
            xi, _, norm = c.xi_window(ell, vs)
            assert relerr(norm * xi.real, d[f"win_xi_{ell}"], FLOOR[form]) < TOL[form], ell


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_zeta_window(form):
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    d = load_golden("xi_window.npz")
    b = binning_from(d["w3_binning"])
    D, R = survey_records(d, "w3")
    vs = float(d["w3_scalars_vsurvey"])
    mps = ((0, 0, 0), (1, 1, 0), (2, 0, 2))
    tol = {"fp64": 1e-10, "fp32": 3e-4}[form]
    with Context(int(d["w3_n_mesh"]), float(d["w3_boxsize"]), b, "TSC", form) as c:
        c.set_particles(1, R, pos_off=survey.POS_OFF, los_off=survey.LOS_OFF, w_off=survey.W_OFF)
        z, sn, norm = c.zeta_window_multi(mps, vs)
        for q, mp in enumerate(mps):
            ref = d["w3_zeta_" + "".join(map(str, mp))]
            assert relerr(norm * (z[q] - sn[q]).real, ref, FLOOR[form]) < tol, mp


def test_window_needs_randoms():
    from hitomi_b200.api import Context, HitomiError
    d = load_golden("xi_window.npz")
    b = binning_from(d["sv_binning"])
    with Context(int(d["sv_n_mesh"]), float(d["sv_boxsize"]), b, "TSC", "fp64") as c:
        with pytest.raises(HitomiError, match="randoms"):
            c.xi_window(0, 1.0e9)
