"""The assignment's fixed-point sums make the density mesh independent of the order in
which the GPU runs its atomics, tiles crowded past one accumulation chunk included: the
bispectrum signal (transforms and fixed-order pair sums downstream of the mesh) is then
bit-identical from run to run, in both forms."""
import numpy as np
import pytest

from conftest import binning_from, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_signal_is_bit_reproducible_with_crowded_tiles(form):
    from hitomi_b200.api import Context
    from hitomi_b200.synthetic import lognormal_box
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    # 60000 particles on a 32^3 mesh: eight tiles of 8 x 16 x 32 cells, ~7500 records each,
    # so every tile is split over several chunks of 2048 records
    pos = lognormal_box(60000, 1000.0, ngrid=32, seed=77, exact_n=60000)
    runs = []
    for _ in range(3):
        with Context(32, 1000.0, b, "TSC", form) as c:
            c.set_particles(0, pos)
            bk, _, _ = c.bk_box_multi(((0, 0, 0), (2, 0, 2)))
            runs.append(bk)
    np.testing.assert_array_equal(runs[0], runs[1])
    np.testing.assert_array_equal(runs[0], runs[2])
