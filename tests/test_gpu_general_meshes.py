"""The correlation-field statistics (bispectrum and 3PCF shot noise, 2PCF) on meshes whose
histograms take the general path -- unequal cells, or a z axis that is not a power of two:
the field transformed whole, folded into octant cells with the reference's per-cell |r|
(field.hpp:1040-1050), Bessel tables at those radii.  Reference outputs from
tests/golden/make_golden.py --general; FP64 1e-10 per bin, FP32 1e-4 of
max(|bin|, 1e-3 max|bins|)."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-10, 1e-12), "fp32": (1e-4, 1e-3)}


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_box_bk_xi_zeta_unequal_cells(form):
    from hitomi_b200.api import Context
    g = load_golden("general_meshes.npz")
    b = binning_from(g["box_binning"])
    tol, floor = TOL[form]
    with Context([int(v) for v in g["box_n_mesh"]], [float(v) for v in g["box_boxsize"]], b, "TSC", form) as c:
        c.set_particles(0, g["box_pos"])
        mps = ((0, 0, 0), (2, 0, 2))
        bk, sn, norm = c.bk_box_multi(mps)
        for q, mp in enumerate(mps):
            assert relerr(norm * (bk[q] - sn[q]), g["box_bk_" + "".join(map(str, mp))], floor) < tol, mp
        for ell in (0, 2):
            xi, nm, xnorm = c.xi_box(ell)
            assert relerr((xnorm * xi).real, g[f"box_xi_{ell}"], floor) < tol, ell
        # the 3PCF on the non-cubic box: j_l(|k| r) at k-space octant keys
        z, zs, zn = c.zeta_box_multi(mps)
        for q, mp in enumerate(mps):
            assert relerr((zn * (z[q] - zs[q])).real, g["box_zeta_" + "".join(map(str, mp))], floor) < tol, mp


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_cubic_mesh_not_power_of_two(form):
    """[48, 48, 48]: equal cells, a 48-point z axis; B (reduced 32-point chain grid) and the
    3PCF, whose shot noise is r-binned from the octant keys."""
    from hitomi_b200.api import Context
    g = load_golden("general_meshes.npz")
    b = binning_from(g["cub_binning"])
    tol, floor = TOL[form]
    with Context(48, 1000.0, b, "TSC", form) as c:
        c.set_particles(0, g["cub_pos"])
        bk, sn, norm = c.bk_box(2, 0, 2)
        assert relerr(norm * (bk - sn), g["cub_bk_202"], floor) < tol
        mps = ((0, 0, 0), (1, 1, 0))
        z, zs, zn = c.zeta_box_multi(mps)
        for q, mp in enumerate(mps):
            assert relerr((zn * (z[q] - zs[q])).real, g["cub_zeta_" + "".join(map(str, mp))], floor) < tol, mp


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_survey_bk_and_xi_unequal_cells(form):
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    g = load_golden("general_meshes.npz")
    b = binning_from(g["sv_binning"])
    L = float(g["sv_boxsize"])
    tol, floor = TOL[form]
    nm = [int(v) for v in g["sv_bk_n_mesh"]]
    D, R = survey.prepare(g["sv_data"], g["sv_rand"], nm, L)
    with Context(nm, L, b, "TSC", form) as c:
        c.set_survey(D, R)
        alpha, vs, *_ = c.survey_scalars()
        mps = ((0, 0, 0), (2, 0, 2))
        bk, sn, norm = c.bk_survey_multi(mps, alpha, vs)
        for q, mp in enumerate(mps):
            assert relerr(norm * (bk[q] - sn[q]), g["sv_bk_" + "".join(map(str, mp))], floor) < tol, mp
    nm = [int(v) for v in g["sv_xi_n_mesh"]]
    D, R = survey.prepare(g["sv_data"], g["sv_rand"], nm, L)
    with Context(nm, L, b, "TSC", form) as c:
        c.set_survey(D, R)
        alpha, vs, *_ = c.survey_scalars()
        for ell in (0, 2):
            xi, _, xnorm = c.xi_survey(ell, alpha, vs)
            assert relerr((xnorm * xi).real, g[f"sv_xi_{ell}"], floor) < tol, ell
