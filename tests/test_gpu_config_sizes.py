"""GPU parity at the configurations' own sizes, against the reference's own code
(tests/golden/make_golden.py --configs, oracle/_ref/ref_harness):

  c1: 2x10^5 uniform particles (seed 1), 1000 Mpc/h box, 128^3 mesh, TSC, P_0,2,4 on 30 bins
      0.005-0.295 h/Mpc (calcPowerSpectrumForBOX, powerspec.hpp:273-332);
  c2: the clustered lognormal catalogue of 10^7 particles (256^3 Gaussian grid, seed 2),
      512^3 mesh, TSC, P_0,2,4 on 25 bins 0.015-0.255 h/Mpc and the B_000 row ith_kbin = 0
      (calcBiSpectrumForBOX, bispec.hpp:877-1203) -- the headline workload.

The catalogues are regenerated from their seeds; their digests (count, coordinate sums and
sums of squares) are checked against the fixture first.  Tolerances, relative to
max(|bin|, 1e-12 max|bins|): the plain FP64 form 1e-10; the chosen form (FP32 with the
density and the bispectrum signal in FP64, hg_config.fp64_stages) 1e-5."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

FORMS = {"fp64": ((), 1e-10), "chosen": (("density", "bk_signal"), 1e-5)}


def digest(pos):
    return np.array([pos.shape[0], *pos.sum(axis=0), *(pos * pos).sum(axis=0)], dtype=np.float64)


def check_digest(pos, ref):
    np.testing.assert_allclose(digest(pos), ref, rtol=1e-12, atol=0)


def context(nm, b, form):
    from hitomi_b200.api import Context
    stages, _ = FORMS[form]
    return Context(nm, 1000.0, b, "TSC", "fp64" if form == "fp64" else "fp32", fp64_stages=stages)


@pytest.fixture(scope="module")
def gold():
    return load_golden("box_config_sizes.npz")


@pytest.mark.parametrize("form", list(FORMS))
def test_config1_pk_128(gold, form):
    from hitomi_b200.synthetic import uniform_box
    pos = uniform_box(200_000, 1000.0, seed=1)
    check_digest(pos, gold["c1_digest"])
    b = binning_from(gold["c1_binning"])
    tol = FORMS[form][1]
    with context(128, b, form) as c:
        c.set_particles(0, pos)
        for ell in (0, 2, 4):
            pk, _, norm = c.pk_box(ell)
            assert relerr(norm * pk, gold[f"c1_pk_{ell}"]) < tol, ell


@pytest.fixture(scope="module")
def c2_catalogue(gold):
    from hitomi_b200.synthetic import lognormal_box
    pos = lognormal_box(10_000_000, 1000.0, ngrid=256, seed=2, exact_n=10_000_000)
    check_digest(pos, gold["c2_digest"])
    return pos


@pytest.mark.parametrize("form", list(FORMS))
def test_config2_pk_and_bk_row_512(gold, c2_catalogue, form):
    b = binning_from(gold["c2_binning"])
    tol = FORMS[form][1]
    with context(512, b, form) as c:
        c.set_particles(0, c2_catalogue)
        for ell in (0, 2, 4):
            pk, _, norm = c.pk_box(ell)
            assert relerr(norm * pk, gold[f"c2_pk_{ell}"]) < tol, ell
        bk, sn, norm = c.bk_box(0, 0, 0, 0)
        assert relerr(norm * (bk[0] - sn[0]), gold["c2_bk000_row0"]) < tol
