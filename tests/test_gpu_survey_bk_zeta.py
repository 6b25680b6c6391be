"""GPU parity of the survey-geometry bispectrum and 3PCF multipoles against the reference
(golden fixtures written by calcBiSpectrum, bispec.hpp:4-352, and
calcThreePointCorrelationFunction, bispec.hpp:355-614, through
tests/golden/make_golden.py --survey3).  (202) and (112) carry M != 0 terms: Yhat_LM-
weighted G fields for every M, conjugate-mirrored fields for M < 0, and azimuth-dependent
shot-noise histograms.  FP64: 1e-10 relative per bin.  FP32: 3e-4 relative to
max(|bin|, 1e-3 max|bins|) -- this catalogue is sparse (2000 galaxies, 32^3 cells), so the
D - alpha R cancellation in every cell amplifies the FP32 rounding of the fields; the
measured errors span 1e-5 to 1.2e-4 from run to run (the accumulation order of the FP32
assignment is not fixed)."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 3e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}
MULTIPOLES = ((0, 0, 0), (1, 1, 0), (2, 0, 2), (1, 1, 2))


def survey_ctx(d, form):
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    b = binning_from(d["binning"])
    nm, bs = int(d["n_mesh"]), float(d["boxsize"])
    D, R = survey.prepare(d["data"], d["rand"], nm, bs)
    c = Context(nm, bs, b, "TSC", form)
    c.set_survey(D, R)
    return c


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_survey_bk_all_multipoles(form):
    d = load_golden("survey_bk_zeta.npz")
    with survey_ctx(d, form) as c:
        alpha, vs, *_ = c.survey_scalars()
        bk, sn, norm = c.bk_survey_multi(MULTIPOLES, alpha, vs)
        for q, mp in enumerate(MULTIPOLES):
            ref = d["bk_" + "".join(map(str, mp))]
            assert relerr(norm * (bk[q] - sn[q]), ref, FLOOR[form]) < TOL[form], mp


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_survey_zeta_all_multipoles(form):
    d = load_golden("survey_bk_zeta.npz")
    with survey_ctx(d, form) as c:
        alpha, vs, *_ = c.survey_scalars()
        z, sn, norm = c.zeta_survey_multi(MULTIPOLES, alpha, vs)
        for q, mp in enumerate(MULTIPOLES):
            ref = d["zeta_" + "".join(map(str, mp))]
            assert relerr(norm * (z[q] - sn[q]).real, ref, FLOOR[form]) < TOL[form], mp


def test_survey_single_rows_and_mixed_calls():
    """One row of one multipole equals that row of the all-rows call; P, B and zeta on the
    same context share the survey fields."""
    d = load_golden("survey_bk_zeta.npz")
    with survey_ctx(d, "fp64") as c:
        alpha, vs, *_ = c.survey_scalars()
        c.pk_survey(2, alpha, vs)
        for ith in (0, 3):
            bk, sn, norm = c.bk_survey(1, 1, 2, alpha, vs, ith)
            assert relerr(norm * (bk[0] - sn[0]), d["bk_112"][ith], 1e-12) < 1e-10
            z, zs, zn = c.zeta_survey(2, 0, 2, alpha, vs, ith)
            assert relerr(zn * (z[0] - zs[0]).real, d["zeta_202"][ith], 1e-12) < 1e-10
