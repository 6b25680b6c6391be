"""BAO reconstruction (hg_reconstruct) and the reconstructed power spectrum against the
reference's drivers (tests/golden/make_golden.py --recon): survey geometry
(calcReconstructionParticles, particle_reconstruction.hpp:12-208, then main.cpp:215-225 and
calcPowerSpectrum with flag_recon) and periodic box (calcReconstructionParticlesForBOX,
:210-402, then main_box.cpp:146-150 and calcPowerSpectrumForBOXForReconstruction,
powerspec.hpp:396-457).  Shifted positions to 1e-9 Mpc/h; P_l to 1e-10 relative per bin
(FP64 form) and 1e-4 of max(|bin|, 1e-3 max|bins|) (FP32 form)."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-10, 1e-12), "fp32": (1e-4, 1e-3)}
POS_TOL = {"fp64": 1e-9, "fp32": 2e-3}


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_survey_reconstruction(form):
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    g = load_golden("recon.npz")
    b = binning_from(g["sv_binning"])
    nm, L, nrec = int(g["sv_n_mesh"]), float(g["sv_boxsize"]), int(g["sv_n_mesh_recon"])
    D, R = survey.prepare(g["sv_data"], g["sv_rand"], nm, L)
    with Context(nm, L, b, "TSC", form) as main, Context(nrec, L, b, "TSC", form) as rc:
        main.set_survey(D, R)
        alpha, vs, *_ = main.survey_scalars()
        rc.set_survey(D, R)
        pD, pR = rc.reconstruct(float(g["sv_b1"]), float(g["sv_RG"]), box=False, alpha=alpha, vsurvey=vs)
        assert np.max(np.abs(pD - g["sv_recon_D"])) < POS_TOL[form]
        assert np.max(np.abs(pR - g["sv_recon_R"])) < POS_TOL[form]
        if form == "fp32":  # continue from the reference's positions: P is compared, not the shift
            pD, pR = g["sv_recon_D"], g["sv_recon_R"]
        D2, R2 = D.copy(), R.copy()
        D2[:, 0:3], R2[:, 0:3] = pD, pR
        survey.shift_into_box(D2, R2, nm, L)  # main.cpp:220
        main.set_survey(D2, R2)
        tol, floor = TOL[form]
        for ell in (0, 2):
            pk, _, norm = main.pk_survey(ell, alpha, vs)
            assert relerr(norm * pk, g[f"sv_pk_{ell}"], floor) < tol, ell


def wrap(p, L):
    """calcPeriodicBoundary (particleGadget.hpp:565-590): one period in or out per axis."""
    q = p.copy()
    q[q >= L] -= L
    q[q < 0.0] += L
    return q


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_box_reconstruction(form):
    from hitomi_b200.api import Context
    g = load_golden("recon.npz")
    b = binning_from(g["box_binning"])
    nm, L, nrec = int(g["box_n_mesh"]), float(g["box_boxsize"]), int(g["box_n_mesh_recon"])
    pos, rnd = g["box_pos"], g["box_rand"]
    with Context(nm, L, b, "TSC", form) as main, Context(nrec, L, b, "TSC", form) as rc:
        rc.set_particles(0, pos)
        rc.set_particles(1, rnd)
        pD, pR = rc.reconstruct(float(g["box_b1"]), float(g["box_RG"]), box=True)
        assert np.max(np.abs(pD - g["box_recon_D"])) < POS_TOL[form]
        assert np.max(np.abs(pR - g["box_recon_R"])) < POS_TOL[form]
        if form == "fp32":
            pD, pR = g["box_recon_D"], g["box_recon_R"]
        main.set_particles(0, wrap(pD, L))
        main.set_particles(1, wrap(pR, L))
        alpha = pos.shape[0] / rnd.shape[0]  # main_box.cpp:150
        tol, floor = TOL[form]
        for ell in (0, 2):
            pk, _, norm = main.pk_box_recon(ell, alpha)
            assert relerr(norm * pk, g[f"box_pk_{ell}"], floor) < tol, ell


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_box_reconstruction_bispectrum_and_3pcf(form):
    """calcBiSpectrumForBOXForReconstruction and
    calcThreePointCorrelationFunctionForBOXForReconstruction (bispec.hpp:1426-1990) on the
    reference's own shifted catalogues, every row."""
    from hitomi_b200.api import Context
    g = load_golden("recon.npz")
    b = binning_from(g["box_bk_binning"])
    nm, L = int(g["box_n_mesh"]), float(g["box_boxsize"])
    alpha = g["box_pos"].shape[0] / g["box_rand"].shape[0]  # main_box.cpp:153
    tol, floor = TOL[form]
    with Context(nm, L, b, "TSC", form) as c:
        c.set_particles(0, wrap(g["box_recon_D"], L))
        c.set_particles(1, wrap(g["box_recon_R"], L))
        mps = ((0, 0, 0), (2, 0, 2))
        bk, sn, norm = c.bk_box_recon_multi(mps, alpha)
        for q, mp in enumerate(mps):
            ref = g["box_bk_" + "".join(map(str, mp))]
            assert relerr(norm * (bk[q] - sn[q]), ref, floor) < tol, mp
        mps = ((0, 0, 0), (1, 1, 0))
        z, zs, znorm = c.zeta_box_recon_multi(mps, alpha)
        for q, mp in enumerate(mps):
            ref = g["box_zeta_" + "".join(map(str, mp))]
            assert relerr((znorm * (z[q] - zs[q])).real, ref, floor) < tol, mp
        # one row alone equals that row of the full matrix
        bk1, sn1, _ = c.bk_box_recon_multi(((2, 0, 2),), alpha, ith_kbin=2)
        assert relerr(bk1[0][0] - sn1[0][0], bk[1][2] - sn[1][2], 1e-12) < 1e-12


def test_reconstruction_needs_both_catalogues():
    from hitomi_b200.api import Context, HitomiError
    g = load_golden("recon.npz")
    b = binning_from(g["box_binning"])
    with Context(32, 1000.0, b, "TSC", "fp64") as c:
        c.set_particles(0, g["box_pos"])
        c._keep[1] = g["box_rand"]
        with pytest.raises(HitomiError, match="randoms"):
            c.reconstruct(1.5, 20.0, box=True)
