"""Meshes whose axes are not powers of two, with unequal cell sizes, against the reference's
own outputs (tests/golden/make_golden.py --mixed): the reference transforms any n_mesh
(FFTW), and its survey meshes (250 x 460 x 260 and the like) are of this kind.  The
transforms of these axes run the mixed-radix pass (radices 4, 2 and odd primes); the
assignment tiles are divisors of each axis.  Tolerances as the other parity tests: FP64
1e-10 per bin, FP32 1e-4 of max(|bin|, 1e-3 max|bins|)."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-10, 1e-12), "fp32": (1e-4, 1e-3)}
POS_TOL = {"fp64": 1e-9, "fp32": 2e-3}


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign", ["TSC", "CIC"])
def test_box_pk_mixed_mesh(form, assign):
    from hitomi_b200.api import Context
    g = load_golden("mixed_meshes.npz")
    b = binning_from(g["box_binning"])
    nm = [int(v) for v in g["box_n_mesh"]]
    bs = [float(v) for v in g["box_boxsize"]]
    tol, floor = TOL[form]
    with Context(nm, bs, b, assign, form) as c:
        c.set_particles(0, g["box_pos"])
        for ell in (0, 2):
            pk, nmode, norm = c.pk_box(ell)
            assert relerr(norm * pk, g[f"box_pk_{assign}_{ell}"], floor) < tol, ell


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_survey_pk_and_reconstruction_mixed_mesh(form):
    """[50, 92, 52] survey mesh (factors 2, 5, 23, 13): the survey scalars and P_l; then the
    reconstruction on a [30, 46, 26] mesh and the reconstructed P_0."""
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    g = load_golden("mixed_meshes.npz")
    b = binning_from(g["sv_binning"])
    nm = [int(v) for v in g["sv_n_mesh"]]
    nrec = [int(v) for v in g["sv_n_mesh_recon"]]
    L = float(g["sv_boxsize"])
    tol, floor = TOL[form]
    D, R = survey.prepare(g["sv_data"], g["sv_rand"], nm, L)
    with Context(nm, L, b, "TSC", form) as main, Context(nrec, L, b, "TSC", form) as rc:
        main.set_survey(D, R)
        alpha, vs, nbar, wd, wr = main.survey_scalars()
        assert abs(alpha - float(g["sv_scalars_alpha"])) <= 1e-12 * abs(float(g["sv_scalars_alpha"]))
        assert abs(vs - float(g["sv_scalars_vsurvey"])) <= 1e-10 * abs(float(g["sv_scalars_vsurvey"]))
        for ell in (0, 2):
            pk, _, norm = main.pk_survey(ell, alpha, vs)
            assert relerr(norm * pk, g[f"sv_pk_{ell}"], floor) < tol, ell
        rc.set_survey(D, R)
        pD, pR = rc.reconstruct(2.0, 40.0, box=False, alpha=alpha, vsurvey=vs)
        assert np.max(np.abs(pD - g["sv_recon_D"])) < POS_TOL[form]
        assert np.max(np.abs(pR - g["sv_recon_R"])) < POS_TOL[form]
        if form == "fp32":  # continue from the reference's positions: P is compared, not the shift
            pD, pR = g["sv_recon_D"], g["sv_recon_R"]
        D2, R2 = D.copy(), R.copy()
        D2[:, 0:3], R2[:, 0:3] = pD, pR
        survey.shift_into_box(D2, R2, nm, L)
        main.set_survey(D2, R2)
        pk, _, norm = main.pk_survey(0, alpha, vs)
        assert relerr(norm * pk, g["sv_recon_pk_0"], floor) < tol


def test_bispectrum_needs_power_of_two_x_when_shells_span_the_axis():
    """When the bispectrum's shells reach the whole of n_mesh_x (4 s + 1 above the reduced
    grid), the fused chain x pass runs on the mesh's own x lines, which must be a power of
    two: the call fails saying so (the 2PCF on the same mesh runs)."""
    from hitomi_b200.api import Context, HitomiError
    g = load_golden("mixed_meshes.npz")
    b = binning_from(g["box_binning"])
    with Context([48, 48, 48], 1000.0, b, "TSC", "fp64") as c:
        c.set_particles(0, g["box_pos"] * np.array([1.0, 1.25, 1.0 / 0.9]))
        assert np.all(np.isfinite(c.pk_box(0)[0]))
        assert np.all(np.isfinite(c.xi_box(0)[0]))
        with pytest.raises(HitomiError, match="power.of.two"):
            c.bk_box(0, 0, 0)


def test_unsupported_meshes_rejected():
    from hitomi_b200.api import Context, HitomiError
    g = load_golden("mixed_meshes.npz")
    b = binning_from(g["box_binning"])
    for nm in ([74, 32, 32], [35, 32, 32], [32, 32, 4096]):  # a prime factor 37; odd; too long
        with pytest.raises(HitomiError):
            Context(nm, 1000.0, b, "TSC", "fp64")
