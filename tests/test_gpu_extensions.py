"""GPU parity of the schemes the reference does not have -- PCS assignment and
interlacing -- against the numpy restatement oracle (oracle/restate.py, pinned to the
reference's own outputs for NGP/CIC/TSC by tests/test_oracle_restate.py); fixtures from
tests/golden/make_golden.py --extensions.  Both use periodic wrap and the exact window
index.  Tolerances as for the reference schemes."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}
CASES = [("PCS", False), ("PCS", True), ("TSC", True), ("CIC", True), ("NGP", True)]


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign,interlace", CASES)
def test_pk_extensions(form, assign, interlace):
    from hitomi_b200.api import Context
    d = load_golden("box_extensions.npz")
    b = binning_from(d["binning"])
    with Context(int(d["n_mesh"]), float(d["boxsize"]), b, assign, form, interlace=interlace) as c:
        c.set_particles(0, d["pos"])
        for ell in (0, 2, 4):
            pk, nmode, norm = c.pk_box(ell)
            np.testing.assert_array_equal(nmode, d[f"nmode_{assign}_{int(interlace)}"])
            assert relerr(norm * pk, d[f"pk_{assign}_{int(interlace)}_{ell}"], FLOOR[form]) < TOL[form], ell


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign,interlace", [("PCS", True), ("TSC", True), ("PCS", False)])
def test_bk_extensions(form, assign, interlace):
    from hitomi_b200.api import Context
    d = load_golden("box_extensions.npz")
    b = binning_from(d["bk_binning"])
    mps = ((0, 0, 0), (1, 1, 0), (2, 0, 2))
    with Context(int(d["n_mesh"]), float(d["boxsize"]), b, assign, form, interlace=interlace) as c:
        c.set_particles(0, d["pos"])
        bk, sn, norm = c.bk_box_multi(mps)
        for q, mp in enumerate(mps):
            ref = d[f"bk_{assign}_{int(interlace)}_" + "".join(map(str, mp))]
            assert relerr(norm * (bk[q] - sn[q]), ref, FLOOR[form]) < TOL[form], mp
