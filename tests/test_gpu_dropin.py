"""The compiled drop-in (hitomi_b200/dropin/hitomi_dropin.hpp): the reference's driver flow
(oracle/ref_harness.cpp, after main_box.cpp:96-228 and main.cpp:129-275) built twice from
the same source -- once with the reference's own estimator bodies (powerspec.hpp,
bispec.hpp), once with the drop-in's bodies over the CUDA library (oracle/Makefile target
`dropin`) -- run on the same parameter file and catalogue.  Both write their files with the
reference's fprintf formats (%.5f / %.7e); the test requires the same file names, the same
header lines, the same k / r columns character for character, and every value equal to the
printed precision (|a - b| <= 6e-8 |b|, half a unit in the eighth significant digit, with a
floor of 1e-9 of the column's largest value for entries that are rounding noise, such as
the imaginary parts of even multipoles).  Plain FP64 form (the default gpu_precision)."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, binning_from, load_golden

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "ref_harness_dropin")


def have_harnesses():
    return all(os.path.exists(p) and os.access(p, os.X_OK) for p in (REF, DROPIN))


def run_both(measure, data, ells, n_mesh, boxsize, b, randoms=None, ith=0, extra="", recon=None, box_recon=False):
    """Run the reference driver and the drop-in driver; return {file name: (ref, dropin) text}."""
    from oracle import ref_runner
    out = {}
    tmp = tempfile.mkdtemp(prefix="hg_dropin_")
    try:
        outs = {}
        for name, exe in (("ref", REF), ("dropin", DROPIN)):
            od = os.path.join(tmp, name, "out")
            os.makedirs(os.path.dirname(od))
            param = os.path.join(tmp, name, "param.ini")
            ref_runner.write_param(param, od, measure, *ells, n_mesh, boxsize, b.kmin, b.kmax, b.n_kbin, b.rmin,
                                   b.rmax, b.n_rbin, "TSC", ith_kbin=ith, ith_rbin=ith, recon=recon)
            if extra:
                with open(param, "a") as f:
                    f.write(extra)
            dpath = os.path.join(tmp, name, "data.f64")
            np.ascontiguousarray(data, dtype=np.float64).tofile(dpath)
            args = [exe, param, dpath] + (["--box-recon"] if box_recon else [])
            if randoms is not None:
                rpath = os.path.join(tmp, name, "random.f64")
                np.ascontiguousarray(randoms, dtype=np.float64).tofile(rpath)
                args.append(rpath)
            env = {k: v for k, v in os.environ.items() if not k.startswith("HX_")}
            p = subprocess.run(args, env=env, capture_output=True, text=True, timeout=600)
            assert p.returncode == 0, (name, p.stdout[-2000:], p.stderr[-2000:])
            outs[name] = od
        names = sorted(f for f in os.listdir(outs["ref"]) if not f.endswith(".f64"))
        assert sorted(f for f in os.listdir(outs["dropin"]) if not f.endswith(".f64")) == names
        for fn in names:
            with open(os.path.join(outs["ref"], fn)) as f1, open(os.path.join(outs["dropin"], fn)) as f2:
                out[fn] = (f1.read(), f2.read())
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return out


def compare_files(files, rel=6e-8, floor_frac=1e-9):
    n_values = 0
    for fn, (a, b) in files.items():
        la, lb = a.splitlines(), b.splitlines()
        assert len(la) == len(lb), fn
        if not fn.endswith(".dat"):
            continue
        assert la[0] == lb[0], fn  # header line
        rows_a = [r.split("\t") for r in la[1:]]
        rows_b = [r.split("\t") for r in lb[1:]]
        ncol = len(rows_a[0])
        # leading k / r columns: identical text; value columns: equal to the printed precision
        nlead = 2 if (fn.startswith("bk") or fn.startswith("zeta")) else 1
        for ra, rb in zip(rows_a, rows_b):
            assert ra[:nlead] == rb[:nlead], fn
        for c in range(nlead, ncol):
            va = np.array([float(r[c]) for r in rows_a])
            vb = np.array([float(r[c]) for r in rows_b])
            floor = floor_frac * float(np.max(np.abs(va))) if va.size else 0.0
            assert np.all(np.abs(vb - va) <= np.maximum(rel * np.abs(va), floor)), (fn, c, va, vb)
            n_values += va.size
    return n_values


@pytest.fixture(autouse=True)
def _need_harnesses():
    if not have_harnesses():
        pytest.fail("oracle/_ref/ref_harness and ref_harness_dropin must be built (make -C oracle all dropin)")


def test_dropin_box_files():
    d = load_golden("xi_window.npz")
    b = binning_from(d["box_binning"])
    pos = d["box_pos"]
    n = 0
    for ell in (0, 2):
        n += compare_files(run_both("pk", pos, (ell, 0, ell), 32, 1000.0, b))
        n += compare_files(run_both("2PCF", pos, (ell, 0, ell), 64, 1000.0, b))
    bb = binning_from(load_golden("box_bk.npz")["binning"])
    for mp in ((0, 0, 0), (2, 0, 2)):
        n += compare_files(run_both("bk", pos, mp, 32, 1000.0, bb, ith=1))
    bz = binning_from(load_golden("box_zeta.npz")["binning"])
    n += compare_files(run_both("3PCF", pos, (1, 1, 0), 32, 1000.0, bz, ith=2))
    assert n > 100


def test_dropin_survey_files():
    g = load_golden("xi_window.npz")
    bs = binning_from(g["sv_binning"])
    data, rand = g["sv_data"], g["sv_rand"]
    n = 0
    n += compare_files(run_both("pk", data, (2, 0, 2), 64, 3500.0, bs, randoms=rand))
    n += compare_files(run_both("2PCF", data, (2, 0, 2), 64, 3500.0, bs, randoms=rand))
    n += compare_files(run_both("window2PCF", data, (2, 0, 2), 64, 3500.0, bs, randoms=rand))
    m = load_golden("mixed_meshes.npz")  # a survey mesh that is not a power of two
    n += compare_files(run_both("pk", m["sv_data"], (2, 0, 2), [int(v) for v in m["sv_n_mesh"]], 3500.0,
                                binning_from(m["sv_binning"]), randoms=m["sv_rand"]))
    b3 = binning_from(g["w3_binning"])
    d3, r3 = g["w3_data"], g["w3_rand"]
    n += compare_files(run_both("bk", d3, (1, 1, 0), 32, 3500.0, b3, randoms=r3, ith=1))
    n += compare_files(run_both("3PCF", d3, (2, 0, 2), 32, 3500.0, b3, randoms=r3, ith=1))
    n += compare_files(run_both("window3PCF", d3, (0, 0, 0), 32, 3500.0, b3, randoms=r3, ith=0))
    assert n > 50


def test_dropin_optional_keys():
    """gpu_precision = chosen runs the FP32 context with FP64 density and bispectrum signal
    (its shot noise in FP32): the files agree with the reference's within that form's bar,
    1e-5 per bin."""
    d = load_golden("box_bk.npz")
    b = binning_from(d["binning"])
    files = run_both("bk", d["pos"], (0, 0, 0), 32, 1000.0, b, ith=3, extra="gpu_precision = chosen\n")
    assert compare_files(files, rel=1e-5, floor_frac=1e-5) > 0


def test_dropin_reconstruction_files():
    """BAO reconstruction through the drop-in (hg_reconstruct on the n_mesh_recon mesh) and
    the estimators that follow it: the survey P with the _recon file name, the box
    reconstructed P, 2PCF, bispectrum and 3PCF."""
    g = load_golden("recon.npz")
    bs = binning_from(g["sv_binning"])
    n = compare_files(run_both("pk", g["sv_data"], (2, 0, 2), 64, 3500.0, bs, randoms=g["sv_rand"],
                               recon=(2.0, 40.0, 32)), rel=1e-7)
    bx = binning_from(g["box_binning"])
    for measure in ("pk", "2PCF"):
        n += compare_files(run_both(measure, g["box_pos"], (0, 0, 0), 32, 1000.0, bx, randoms=g["box_rand"],
                                    recon=(1.5, 20.0, 32), box_recon=True), rel=1e-7)
    bb = binning_from(g["box_bk_binning"])
    for measure, mp in (("bk", (2, 0, 2)), ("3PCF", (1, 1, 0))):
        n += compare_files(run_both(measure, g["box_pos"], mp, 32, 1000.0, bb, randoms=g["box_rand"],
                                    recon=(1.5, 20.0, 32), box_recon=True, ith=1), rel=1e-7)
    assert n > 30
