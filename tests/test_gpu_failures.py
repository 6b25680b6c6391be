"""Failure handling on the host, with no GPU fault: catalogues with non-finite or far-away
positions, particles outside the box (against the reference's own outputs), a device memory
limit that makes an allocation fail on purpose, and a batch that stops at a failing mock.
Every failure here is detected on the host or by a count the kernels keep; nothing traps."""
import numpy as np
import pytest

from conftest import binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}


def ctx_for(d, form="fp64", assign="TSC", **kw):
    from hitomi_b200.api import Context
    return Context(int(d["n_mesh"]), float(d["boxsize"]), binning_from(d["binning"]), assign, form, **kw)


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_nonfinite_position_rejected_and_context_usable(form, bad):
    from hitomi_b200.api import HitomiError
    d = load_golden("box_bk.npz")
    pos = d["pos"].copy()
    pos[123, 1] = bad
    with ctx_for(d, form) as c:
        c.set_particles(0, pos)
        with pytest.raises(HitomiError, match="non-finite"):
            c.pk_box(0)
        with pytest.raises(HitomiError, match="non-finite"):
            c.bk_box_multi(((0, 0, 0),))
        c.set_particles(0, d["pos"])  # the same context, a valid catalogue
        pk, nm, norm = c.pk_box(0)
        bk, sn, bnorm = c.bk_box_multi(((0, 0, 0),))
    with ctx_for(d, form) as c:
        c.set_particles(0, d["pos"])
        pk2, nm2, norm2 = c.pk_box(0)
        bk2, sn2, _ = c.bk_box_multi(((0, 0, 0),))
    # P's bin sums add with FP64 atomics (last-bit order dependence); the signal is exact
    assert relerr(pk, pk2) < 1e-14
    np.testing.assert_array_equal(nm, nm2)
    np.testing.assert_array_equal(bk, bk2)


def test_nonfinite_survey_weight_rejected():
    from hitomi_b200 import survey
    from hitomi_b200.api import HitomiError
    from hitomi_b200.api import Context
    g = load_golden("survey_pk.npz")
    b = binning_from(g["binning"])
    nm, bs = int(g["n_mesh"]), float(g["boxsize"])
    data, rand = survey.prepare(g["data"], g["rand"], nm, bs)
    for which in (0, 1):
        dd, rr = data.copy(), rand.copy()
        (dd if which == 0 else rr)[7, survey.W_OFF] = np.nan
        with Context(nm, bs, b, "TSC", "fp64") as c:
            c.set_survey(dd, rr)
            with pytest.raises(HitomiError, match="non-finite"):
                c.survey_scalars()


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("assign", ["NGP", "CIC", "TSC"])
def test_outside_box_matches_reference(form, assign):
    """A quarter of the particles within 1.6 cells beyond a face and a few up to three box
    lengths away: the reference's int() truncation and flat-index rule (its own outputs)."""
    d = load_golden("box_outside.npz")
    with ctx_for(d, form, assign) as c:
        c.set_particles(0, d["pos"])
        for ell in (0, 2):
            pk, nm, norm = c.pk_box(ell)
            assert relerr(norm * pk, d[f"pk_{assign}_{ell}"], FLOOR[form]) < TOL[form], ell
        bk, sn, norm = c.bk_box_multi(((0, 0, 0),))
        assert relerr(norm * (bk[0] - sn[0]), d[f"bk_{assign}_000"], FLOOR[form]) < TOL[form]


@pytest.mark.parametrize("assign", ["CIC", "TSC"])
def test_far_positions_are_dropped(assign):
    """Coordinates 10^12 box lengths away on one axis (beyond the int range of the anchor)
    give exactly what particles 100 box lengths away on every axis give -- a flat index far
    past the mesh under the reference's rule, so no cell -- with the same particle count.
    (100 box lengths on the z axis alone would not do: the flat-index rule carries z into
    y and x, and such a particle lands in the mesh.)"""
    d = load_golden("box_bk.npz")
    L = float(d["boxsize"])
    out = {}
    for far in (None, 1e12 * L):
        pos = d["pos"].copy()
        if far is None:
            pos[:6] = 100.0 * L
        else:
            pos[:6] = [[far, 10.0, 10.0], [-far, 10.0, 10.0], [10.0, far, 10.0], [10.0, -far, 10.0],
                       [10.0, 10.0, far], [10.0, 10.0, -far]]
        with ctx_for(d, "fp64", assign) as c:
            c.set_particles(0, pos)
            out[far] = (c.pk_box(0), c.bk_box_multi(((0, 0, 0),)))
    (pa, ba), (pb, bb) = out.values()
    assert relerr(pa[0], pb[0]) < 1e-14
    np.testing.assert_array_equal(pa[1], pb[1])
    np.testing.assert_array_equal(ba[0], bb[0])
    assert relerr(ba[1], bb[1]) < 1e-12


def test_far_positions_wrap_on_periodic_mesh():
    """PCS (periodic wrap): a coordinate 2^40 box lengths away is reduced into the box
    (x - L floor(x / L)) before assignment, as the same reduction done here gives."""
    d = load_golden("box_bk.npz")
    L = float(d["boxsize"])
    pos = d["pos"].copy()
    pos[:50, 0] += L * 2.0 ** 40
    red = pos.copy()
    red[:50, 0] = red[:50, 0] - L * np.floor(red[:50, 0] / L)
    res = []
    for p in (pos, red):
        with ctx_for(d, "fp64", "PCS") as c:
            c.set_particles(0, p)
            res.append(c.pk_box(0)[0])
    assert relerr(res[0], res[1]) < 1e-14


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_memory_limit_fails_then_recovers(form):
    from hitomi_b200.api import HitomiError
    d = load_golden("box_bk.npz")
    with ctx_for(d, form) as c:
        c.set_particles(0, d["pos"])
        c.set_memory_limit(1 << 20)
        with pytest.raises(HitomiError, match="memory limit"):
            c.bk_box_multi(((0, 0, 0), (2, 0, 2)))
        assert c.memory_in_use() <= 1 << 20
        with pytest.raises(HitomiError):
            c.set_memory_limit(-1)
        c.set_memory_limit(0)
        bk, sn, norm = c.bk_box_multi(((0, 0, 0), (2, 0, 2)))
        assert c.memory_in_use() > 1 << 20
        held = c.memory_in_use()
        c.set_memory_limit(held)  # everything it needs is held: runs again within the cap
        bk2, sn2, _ = c.bk_box_multi(((0, 0, 0), (2, 0, 2)))
    np.testing.assert_array_equal(bk, bk2)
    for q, mp in enumerate(((0, 0, 0), (2, 0, 2))):
        ref = d["bk_TSC_" + "".join(map(str, mp))]
        assert relerr(norm * (bk[q] - sn[q]), ref, FLOOR[form]) < TOL[form]


def test_batch_stops_at_failing_mock():
    """Mock 1 of 3 holds a NaN position: the batch reports mock 1, mock 0's block is complete
    and equals a single call, and the context then runs the remaining mocks."""
    from hitomi_b200.api import BatchError
    d = load_golden("box_bk.npz")
    good = d["pos"]
    bad = good.copy()
    bad[5, 2] = np.nan
    other = good[::-1].copy() * 0.5
    with ctx_for(d, "fp64") as c:
        with pytest.raises(BatchError, match="mock 1") as ei:
            c.batch_run([good, bad, other], pk_ells=(0, 2), bk_multipoles=((0, 0, 0),))
        assert ei.value.done == 1 and len(ei.value.results) == 1
        r0 = ei.value.results[0]
        rest = c.batch_run([other], pk_ells=(0, 2), bk_multipoles=((0, 0, 0),))
        c.set_particles(0, good)
        pk0 = c.pk_box(0)[0]
        bk0 = c.bk_box_multi(((0, 0, 0),))[0]
        c.set_particles(0, other)
        pko = c.pk_box(0)[0]
    assert relerr(r0["pk"][0], pk0) < 1e-14
    np.testing.assert_array_equal(r0["bk"], bk0)
    assert relerr(rest[0]["pk"][0], pko) < 1e-14


def test_empty_catalogue_rejected():
    """Zero particles: the reference's message (particle.hpp:50-53); the context keeps its
    previous catalogue."""
    from hitomi_b200.api import HitomiError
    d = load_golden("box_bk.npz")
    with ctx_for(d, "fp64") as c:
        c.set_particles(0, d["pos"])
        with pytest.raises(HitomiError, match="should be > 0"):
            c.set_particles(0, np.zeros((0, 3)))
        assert np.all(np.isfinite(c.pk_box(0)[0]))
