"""Every launch shape of the fused chain x pass (kChainVariants, hg_fft2.cuh) gives the same
bispectrum.  The autotuner keeps whichever variant is fastest on the first mock, so each one
must be exact; HG_CHAIN_VARIANT forces one variant untimed.  256^3 mesh, shells to |n| = 35:
the chains run on the 192^3 reduced grid, where all fifteen variants exist.  Reference
values from the numpy restatement pinned to the reference; tolerances as the other parity
tests."""
import os

import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}
N_VARIANTS = 15


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_every_chain_variant(form):
    from hitomi_b200.api import Context
    d = load_golden("box_bk_256.npz")
    b = binning_from(d["binning"])
    try:
        for v in range(N_VARIANTS):
            os.environ["HG_CHAIN_VARIANT"] = str(v)
            with Context(256, float(d["boxsize"]), b, "TSC", form) as c:
                c.set_particles(0, d["pos"])
                bk, sn, norm = c.bk_box(0, 0, 0)
                assert f"variant {v} " in c.tuning(), c.tuning()
            assert relerr(norm * (bk - sn), d["bk_000"], FLOOR[form]) < TOL[form], v
    finally:
        os.environ.pop("HG_CHAIN_VARIANT", None)


def test_unknown_chain_variant_rejected():
    from hitomi_b200.api import Context, HitomiError
    d = load_golden("box_bk_256.npz")
    b = binning_from(d["binning"])
    try:
        os.environ["HG_CHAIN_VARIANT"] = str(N_VARIANTS)
        with Context(256, float(d["boxsize"]), b, "TSC", "fp64") as c:
            c.set_particles(0, d["pos"])
            with pytest.raises(HitomiError, match="HG_CHAIN_VARIANT"):
                c.bk_box(0, 0, 0)
    finally:
        os.environ.pop("HG_CHAIN_VARIANT", None)
