"""hg_batch_run: many catalogues in one call, the next one's upload overlapping the current
one's statistics.  Each mock's block must equal what the single-catalogue entry points give
(hg_pk_box, hg_bk_box_multi, hg_zeta_box_multi), for catalogues of different sizes and
record layouts, in both forms."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

MULTIPOLES = ((0, 0, 0), (2, 0, 2))
ZETA = ((0, 0, 0), (1, 1, 0))


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_batch_equals_single_calls(form):
    from hitomi_b200.api import Context
    from hitomi_b200.synthetic import lognormal_box
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    mocks = [lognormal_box(n, 1000.0, ngrid=32, seed=40 + i, exact_n=n) for i, n in enumerate((9000, 15000, 4000))]
    # the second mock as {pos, vel} records (48-byte stride)
    g = np.zeros((mocks[1].shape[0], 6))
    g[:, :3] = mocks[1]
    g[:, 3:] = -7.0
    mocks[1] = g
    # two runs of the same catalogue agree to the order-dependent last bits of the FP64 atomics
    # (FP64 form) or of the FP32 float atomics of crowded assignment tiles (FP32 form)
    tol = {"fp64": 1e-10, "fp32": 1e-5}[form]
    with Context(32, 1000.0, b, "TSC", form) as c:
        res = c.batch_run(mocks, pk_ells=(0, 2), bk_multipoles=MULTIPOLES, zeta_multipoles=ZETA)
        assert len(res) == 3
        for m, r in zip(mocks, res):
            c.set_particles(0, m)
            for q, ell in enumerate((0, 2)):
                pk, _, norm = c.pk_box(ell)
                assert relerr(r["pk"][q], pk, 1e-3) < tol and r["pk_norm"][q] == norm
            bk, sn, norm = c.bk_box_multi(MULTIPOLES)
            assert relerr(r["bk"], bk, 1e-3) < tol and relerr(r["bk_sn"], sn, 1e-3) < tol and r["bk_norm"] == norm
            z, zs, zn = c.zeta_box_multi(ZETA)
            assert relerr(r["zeta"], z, 1e-3) < tol and relerr(r["zeta_sn"], zs, 1e-3) < tol and r["zeta_norm"] == zn


def test_batch_rejects_bad_mocks():
    from hitomi_b200.api import Context, HitomiError
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    with Context(32, 1000.0, b, "TSC", "fp64") as c:
        with pytest.raises(HitomiError):
            c.batch_run([np.zeros((0, 3))], pk_ells=(0,))
        with pytest.raises(HitomiError, match="not allowed"):
            c.batch_run([d["pos"]], bk_multipoles=((1, 0, 0),))
