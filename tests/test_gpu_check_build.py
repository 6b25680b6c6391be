"""The check build (libhitomi_b200_check.so, -DHG_CHECK): device-side bounds checks at the
index-sensitive accesses -- particle records inside their tile's range, stencil points
inside the CTA's tile, mesh cells inside the mesh, coarse bins inside the binning arrays,
chain rows inside the kept cube, mixed-radix line indices -- each recording the first
failure and skipping the access, the call failing afterwards.  The reference fixtures run
through it: every call succeeds (no check fails) and gives what the normal build gives."""
import os

import numpy as np
import pytest

from conftest import ROOT, binning_from, load_golden, relerr

pytestmark = pytest.mark.gpu

CHECK_LIB = os.path.join(ROOT, "hitomi_b200", "libhitomi_b200_check.so")


@pytest.fixture(autouse=True)
def _need_check_build():
    if not os.path.exists(CHECK_LIB):
        pytest.fail("the check build is missing: python hitomi_b200/build.py --check")


def both(make, run):
    out = []
    for check in (False, True):
        with make(check) as c:
            out.append(run(c))
    return out


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_box_pk_bk_zeta(form):
    from hitomi_b200.api import Context
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    mps = ((0, 0, 0), (1, 1, 0), (2, 0, 2))

    def run(c):
        c.set_particles(0, d["pos"])
        return c.pk_box(2)[0], c.bk_box_multi(mps)[:2]

    (p0, (b0, s0)), (p1, (b1, s1)) = both(
        lambda ck: Context(int(d["n_mesh"]), float(d["boxsize"]), b, "TSC", form, check_build=ck), run)
    assert relerr(p1, p0) < 1e-12
    np.testing.assert_array_equal(b1, b0)  # the signal is exact in both builds
    assert relerr(s1, s0) < 1e-10
    z = load_golden("box_zeta.npz")
    bz = binning_from(z["binning"])

    def runz(c):
        c.set_particles(0, z["pos"])
        return c.zeta_box_multi(((0, 0, 0), (1, 1, 0)))[:2]

    (z0, zs0), (z1, zs1) = both(
        lambda ck: Context(int(z["n_mesh"]), float(z["boxsize"]), bz, "TSC", form, check_build=ck), runz)
    assert relerr(z1, z0) < 1e-12 and relerr(zs1, zs0) < 1e-10


def test_edges_outside_and_mixed_meshes():
    """The flat-index rule's edge particles, particles outside the box, and a mesh that is
    not a power of two (mixed-radix transforms, dividing tiles)."""
    from hitomi_b200.api import Context
    for name in ("box_edges.npz", "box_outside.npz"):
        d = load_golden(name)
        b = binning_from(d["binning"])
        for assign in ("NGP", "CIC", "TSC"):
            def run(c):
                c.set_particles(0, d["pos"])
                return c.pk_box(0)[0], c.bk_box(0, 0, 0)[0]

            (p0, b0), (p1, b1) = both(
                lambda ck: Context(int(d["n_mesh"]), float(d["boxsize"]), b, assign, "fp64", check_build=ck), run)
            assert relerr(p1, p0) < 1e-12
            np.testing.assert_array_equal(b1, b0)
    m = load_golden("mixed_meshes.npz")
    bm = binning_from(m["box_binning"])

    def runm(c):
        c.set_particles(0, m["box_pos"])
        return c.pk_box(2)[0]

    q0, q1 = both(lambda ck: Context([int(v) for v in m["box_n_mesh"]], [float(v) for v in m["box_boxsize"]], bm,
                                     "TSC", "fp64", check_build=ck), runm)
    assert relerr(q1, q0) < 1e-12


def test_survey():
    from hitomi_b200 import survey
    from hitomi_b200.api import Context
    g = load_golden("survey_bk_zeta.npz")
    b = binning_from(g["binning"])
    nm, L = int(g["n_mesh"]), float(g["boxsize"])
    D, R = survey.prepare(g["data"], g["rand"], nm, L)

    def run(c):
        c.set_survey(D, R)
        alpha, vs, *_ = c.survey_scalars()
        return c.pk_survey(2, alpha, vs)[0], c.bk_survey_multi(((2, 0, 2),), alpha, vs)[0]

    (p0, b0), (p1, b1) = both(lambda ck: Context(nm, L, b, "TSC", "fp64", check_build=ck), run)
    assert relerr(p1, p0) < 1e-12
    assert relerr(b1, b0) < 1e-12
