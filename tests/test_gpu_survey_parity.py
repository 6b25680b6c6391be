"""GPU parity of the survey-geometry (Yamamoto, local line of sight) power-spectrum
multipoles and survey scalars against the reference (golden fixtures written by
calcPowerSpectrum, powerspec.hpp:4-91, and the survey driver main.cpp:129-200, through
tests/golden/make_golden.py).

The catalogues are prepared exactly as the reference's driver does
(hitomi_b200.survey.prepare: LOS, shift into the FFT box), so the library sees the same
records.  Tolerances: FP64 1e-10 relative per bin; FP32 1e-4 relative to
max(|bin|, 1e-3 max|bins|); the scalars are FP64 in both forms."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}


def survey_ctx(d, assign, form):
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    b = binning_from(d["binning"])
    nm, bs = int(d["n_mesh"]), float(d["boxsize"])
    D, R = survey.prepare(d["data"], d["rand"], nm, bs)
    c = Context(nm, bs, b, assign, form)
    c.set_survey(D, R)
    return c


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign", ["NGP", "CIC", "TSC"])
def test_survey_scalars(form, assign):
    d = load_golden("survey_pk.npz")
    with survey_ctx(d, assign, form) as c:
        alpha, vs, nbar, wd, wr = c.survey_scalars()
    for name, v in (("alpha", alpha), ("vsurvey", vs), ("nbar", nbar), ("wsum_data", wd), ("wsum_rand", wr)):
        ref = float(d[f"scalars_{assign}_{name}"])
        assert abs(v - ref) <= 1e-12 * abs(ref), name


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_survey_pk_all_ells_tsc(form):
    d = load_golden("survey_pk.npz")
    with survey_ctx(d, "TSC", form) as c:
        alpha, vs, *_ = c.survey_scalars()
        for ell in (0, 1, 2, 3, 4):
            pk, nmode, norm = c.pk_survey(ell, alpha, vs)
            assert relerr(norm * pk, d[f"pk_TSC_{ell}"], FLOOR[form]) < TOL[form], ell


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign", ["NGP", "CIC"])
def test_survey_pk_other_assignments(form, assign):
    d = load_golden("survey_pk.npz")
    with survey_ctx(d, assign, form) as c:
        alpha, vs, *_ = c.survey_scalars()
        for ell in (0, 2):
            pk, nmode, norm = c.pk_survey(ell, alpha, vs)
            assert relerr(norm * pk, d[f"pk_{assign}_{ell}"], FLOOR[form]) < TOL[form], ell


def test_survey_repeat_and_alpha_change():
    """Fields are cached per alpha: a second call with the same alpha reuses them, a
    different alpha rebuilds them (the result scales the randoms' share)."""
    d = load_golden("survey_pk.npz")
    with survey_ctx(d, "TSC", "fp64") as c:
        alpha, vs, *_ = c.survey_scalars()
        p1, _, n1 = c.pk_survey(2, alpha, vs)
        p2, _, n2 = c.pk_survey(2, alpha, vs)
        np.testing.assert_allclose(p1, p2, rtol=1e-12, atol=1e-12 * np.abs(p1).max())
        p3, _, _ = c.pk_survey(2, 1.1 * alpha, vs)
        assert np.abs(p3 - p1).max() > 1e-6 * np.abs(p1).max()
        p4, _, _ = c.pk_survey(2, alpha, vs)
        np.testing.assert_allclose(p4, p1, rtol=1e-12, atol=1e-12 * np.abs(p1).max())
        assert relerr(n1 * p1, d["pk_TSC_2"], 1e-12) < 1e-10


def test_survey_errors():
    from hitomi_b200.api import Binning, Context, HitomiError
    d = load_golden("survey_pk.npz")
    b = binning_from(d["binning"])
    with Context(32, 3500.0, b, "TSC", "fp64") as c:
        with pytest.raises(HitomiError, match="randoms"):
            c.survey_scalars()
        from hitomi_b200 import survey
        D, R = survey.prepare(d["data"], d["rand"], 32, 3500.0)
        c.set_particles(0, D, w_off=6)
        c.set_particles(1, R, w_off=6)
        c.survey_scalars()  # no LOS needed
        with pytest.raises(HitomiError, match="line-of-sight"):
            c.pk_survey(2, 0.05, 1e9)
