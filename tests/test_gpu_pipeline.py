"""Two contexts on one GPU driven from two host threads (hitomi_b200.batch.run_pipelined)
give the same statistics as one context used mock after mock."""
import numpy as np
import pytest

from conftest import binning_from, load_golden

pytestmark = pytest.mark.gpu


def test_pipelined_contexts_match_sequential():
    from hitomi_b200.api import Context
    from hitomi_b200.batch import run_pipelined

    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    rng = np.random.default_rng(7)
    mocks = [np.ascontiguousarray(d["pos"][rng.permutation(d["pos"].shape[0])[:9000]]) for _ in range(5)]

    def measure_on(c, i):
        c.set_particles(0, mocks[i])
        pk, _, norm = c.pk_box(0)
        bk, sn, bnorm = c.bk_box(0, 0, 0)
        return {"pk": norm * pk, "bk": bnorm * (bk - sn)}

    args = (int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", "fp64")
    with Context(*args) as c:
        seq = {i: measure_on(c, i) for i in range(len(mocks))}
    with Context(*args) as c1, Context(*args) as c2:
        par = run_pipelined(list(range(len(mocks))), [c1, c2], measure_on)
    for i in range(len(mocks)):
        for k in ("pk", "bk"):
            np.testing.assert_allclose(par[i][k], seq[i][k], rtol=1e-12, atol=0)
