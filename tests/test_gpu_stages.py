"""FP32 contexts that run chosen stages of the periodic-box pipeline in FP64
(hg_config.fp64_stages): the FP64 stages must give what the plain FP64 form gives, and
every combination must still match the reference's fixtures."""
import itertools

import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

MULTIPOLES = ((0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2))
STAGES = ("density", "bk_signal", "bk_shot")


def run(form, stages, d, b):
    from hitomi_b200.api import Context
    with Context(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", form, fp64_stages=stages) as c:
        c.set_particles(0, d["pos"])
        pk = {ell: c.pk_box(ell) for ell in (0, 2, 4)}
        bk, sn, norm = c.bk_box_multi(MULTIPOLES)
        return pk, (bk, sn, norm)


def test_all_stages_fp64_equals_plain_form():
    """With every stage in FP64 the FP32 context computes exactly what the FP64 form does
    (same kernels on the same FP64 data)."""
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    pk64, (bk64, sn64, n64) = run("fp64", (), d, b)
    pkm, (bkm, snm, nm) = run("fp32", STAGES, d, b)
    for ell in (0, 2, 4):
        assert relerr(pkm[ell][0], pk64[ell][0]) < 1e-13, ell
        np.testing.assert_array_equal(pkm[ell][1], pk64[ell][1])
    assert nm == n64
    assert relerr(bkm, bk64) < 1e-13
    # the shot-noise histogram adds with FP64 atomics: order-dependent at the last bits,
    # which the cancellation between its terms lifts to ~1e-12 of a bin
    assert relerr(snm, sn64) < 1e-11


@pytest.mark.parametrize("stages", [s for r in range(1, 3) for s in itertools.combinations(STAGES, r)])
def test_stage_combinations_match_reference(stages):
    """Every partial set of FP64 stages still reproduces the reference's B and P fixtures at
    the FP32 form's tolerance (1e-4 of max(|bin|, 1e-3 max|bins|) on these sparse catalogues),
    and the stages run in FP64 come out at the FP64 form's values."""
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    pk, (bk, sn, norm) = run("fp32", stages, d, b)
    for q, mp in enumerate(MULTIPOLES):
        ref = d["bk_TSC_" + "".join(map(str, mp))]
        assert relerr(norm * (bk[q] - sn[q]), ref, 1e-3) < 1e-4, (stages, mp)
    if "density" in stages:  # P_l is binned from the FP64 spectrum
        pk64, _ = run("fp64", (), d, b)
        for ell in (0, 2, 4):
            assert relerr(pk[ell][0], pk64[ell][0]) < 1e-13, ell


def test_stage_kernels_are_reported():
    """Profiling lists the FP64 stages' kernels under an fp64: prefix."""
    from hitomi_b200.api import Context
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    with Context(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", "fp32", fp64_stages=("bk_shot",)) as c:
        c.set_particles(0, d["pos"])
        c.set_profiling(True)
        c.bk_box_multi(MULTIPOLES)
        st = c.kernel_stats()
        assert any(k.startswith("fp64:xi_") for k in st), sorted(st)
        assert any(k.startswith("chain_") for k in st), sorted(st)
        assert c.last_timing()[1] > 0


def test_unknown_stage_bits_rejected():
    from hitomi_b200.api import Context, HitomiError
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    with pytest.raises(HitomiError, match="fp64_stages"):
        Context(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", "fp32", fp64_stages=64)
