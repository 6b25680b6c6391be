"""Regenerate the golden fixtures in tests/golden/ from the CPU oracle.

The values come from oracle/_ref/ref_harness: the reference's own estimator headers
(src/hitomi_measurement/*.hpp) compiled against the project's FFTW/GSL shims, run
with 17-significant-digit output.  Inputs are stored in the fixture next to the outputs
so the GPU tests need neither the reference sources nor the harness.

    python tests/golden/make_golden.py          (needs `make -C oracle` first)
    python tests/golden/make_golden.py --zeta   (only box_zeta.npz)
    python tests/golden/make_golden.py --survey (only survey_pk.npz)
    python tests/golden/make_golden.py --survey3 (only survey_bk_zeta.npz)
    python tests/golden/make_golden.py --odd (only box_odd.npz: odd l1 + l2)
    python tests/golden/make_golden.py --bk256 (only box_bk_256.npz, from the restatement)
    python tests/golden/make_golden.py --xi     (only xi_window.npz: 2PCF, window 2PCF / 3PCF)
    python tests/golden/make_golden.py --ingest (only ingest.npz: the ASCII and Gadget readers)
    python tests/golden/make_golden.py --recon  (only recon.npz: BAO reconstruction)
    python tests/golden/make_golden.py --outside (only box_outside.npz: particles outside the box)
    python tests/golden/make_golden.py --long   (only box_long_axes.npz: 1024-point axes)
    python tests/golden/make_golden.py --mixed  (only mixed_meshes.npz: non-power-of-two meshes)
    python tests/golden/make_golden.py --general (only general_meshes.npz: B, 2PCF, 3PCF on such meshes)
    python tests/golden/make_golden.py --configs (only box_config_sizes.npz: 128^3 and 512^3)
    python tests/golden/make_golden.py --extensions (only box_extensions.npz: PCS and
        interlacing, from the numpy restatement oracle/restate.py; no harness needed)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hitomi_b200.api import Binning  # noqa: E402
from hitomi_b200.synthetic import lognormal_box, survey_shell, uniform_box  # noqa: E402
from oracle import ref_runner  # noqa: E402

MULTIPOLES = ((0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2))
ZETA_MULTIPOLES = ((0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2), (1, 1, 2))
SURVEY_MULTIPOLES = ((0, 0, 0), (1, 1, 0), (2, 0, 2), (1, 1, 2))


def binning_arr(b: Binning):
    return np.array([b.kmin, b.kmax, b.n_kbin, b.rmin, b.rmax, b.n_rbin], dtype=np.float64)


def edge_catalogue(n_mesh: int, boxsize: float, n: int, seed: int) -> np.ndarray:
    """Particles concentrated on cell edges and on the box faces, where the reference's
    flat-index rule (field.hpp:92-96) drops or moves stencil points."""
    rng = np.random.default_rng(seed)
    dr = boxsize / n_mesh
    pos = rng.uniform(0.0, boxsize, size=(n, 3))
    k = n // 3
    # on cell edges and half-cell points
    pos[:k] = np.floor(pos[:k] / dr) * dr + rng.choice([0.0, 0.5 * dr, 1e-9, dr - 1e-9], size=(k, 3))
    # hugging the upper and lower faces
    face = rng.integers(0, 3, size=k)
    side = rng.random(k) < 0.5
    vals = np.where(side, boxsize - rng.uniform(0.0, 0.75 * dr, k), rng.uniform(0.0, 0.75 * dr, k))
    pos[k:2 * k][np.arange(k), face] = vals
    pos = np.clip(pos, 0.0, np.nextafter(boxsize, 0.0))
    return np.ascontiguousarray(pos)


def run_pk(pos, n_mesh, boxsize, b, assign, ells=(0, 2, 4)):
    out = {}
    for ell in ells:
        with ref_runner.RefRun() as r:
            r.run("pk", pos, ell, 0, ell, n_mesh, boxsize, b, assign=assign)
            out[ell] = r.pk(ell)[1]
    return out


def run_bk(pos, n_mesh, boxsize, b, assign, mps=MULTIPOLES):
    out = {}
    for mp in mps:
        with ref_runner.RefRun() as r:
            r.run("bk", pos, *mp, n_mesh, boxsize, b, assign=assign)
            out[mp] = r.bk(*mp, b.n_kbin)
    return out


def run_zeta(pos, n_mesh, boxsize, b, assign, mps=ZETA_MULTIPOLES):
    out = {}
    for mp in mps:
        with ref_runner.RefRun() as r:
            r.run("3PCF", pos, *mp, n_mesh, boxsize, b, assign=assign)
            out[mp] = r.zeta(*mp, b.n_rbin)
    return out


def make_zeta():
    """3PCF multipoles, all rows: file values norm * Re(zeta - sn) (bispec.hpp:1402-1416)."""
    pos = lognormal_box(10000, 400.0, ngrid=32, seed=15, exact_n=10000)
    bz = Binning(0.02, 0.1, 5, 20.0, 140.0, 7)
    d = dict(pos=pos, boxsize=400.0, n_mesh=32, binning=binning_arr(bz))
    for mp, v in run_zeta(pos, 32, 400.0, bz, "TSC").items():
        d["zeta_TSC_" + "".join(map(str, mp))] = v
    for assign in ("NGP", "CIC"):
        for mp, v in run_zeta(pos, 32, 400.0, bz, assign, mps=((0, 0, 0),)).items():
            d[f"zeta_{assign}_" + "".join(map(str, mp))] = v
    # r bins reaching past half the box and below one cell, on the boundary-stress catalogue
    pe = edge_catalogue(16, 400.0, 6000, seed=13)
    be = Binning(0.02, 0.1, 5, 10.0, 250.0, 9)
    d["edge_pos"] = pe
    d["edge_binning"] = binning_arr(be)
    d["edge_zeta_TSC_000"] = run_zeta(pe, 16, 400.0, be, "TSC", mps=((0, 0, 0),))[(0, 0, 0)]
    d["edge_zeta_TSC_110"] = run_zeta(pe, 16, 400.0, be, "TSC", mps=((1, 1, 0),))[(1, 1, 0)]
    np.savez_compressed(os.path.join(HERE, "box_zeta.npz"), **d)


def make_survey():
    """Survey-geometry P_l (powerspec.hpp:4-91) and the survey scalars (main.cpp:150-200),
    on a shell-and-cap catalogue; every assignment for l = 0, 2 and one scheme for all l."""
    data, rand = survey_shell(3000, 60000, seed=16)
    bs = Binning(0.004, 0.048, 12, 20.0, 140.0, 7)
    d = dict(data=data, rand=rand, boxsize=3500.0, n_mesh=64, binning=binning_arr(bs))
    for assign, ells in (("TSC", (0, 1, 2, 3, 4)), ("CIC", (0, 2)), ("NGP", (0, 2))):
        for ell in ells:
            with ref_runner.RefRun() as r:
                r.run("pk", data, ell, 0, ell, 64, 3500.0, bs, assign=assign, randoms=rand)
                d[f"pk_{assign}_{ell}"] = r.pk(ell)[1]
                sc = r.survey_scalars()
        for k, v in sc.items():
            d[f"scalars_{assign}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "survey_pk.npz"), **d)


def make_survey_three_point():
    """Survey-geometry bispectrum (bispec.hpp:4-352) and 3PCF (bispec.hpp:355-614)
    multipoles, all rows; (202) and (112) have M != 0 terms."""
    data, rand = survey_shell(2000, 30000, seed=18)
    b = Binning(0.004, 0.02, 5, 150.0, 750.0, 5)
    d = dict(data=data, rand=rand, boxsize=3500.0, n_mesh=32, binning=binning_arr(b))
    for mp in SURVEY_MULTIPOLES:
        tag = "".join(map(str, mp))
        with ref_runner.RefRun() as r:
            r.run("bk", data, *mp, 32, 3500.0, b, assign="TSC", randoms=rand)
            d["bk_" + tag] = r.bk(*mp, b.n_kbin)
        with ref_runner.RefRun() as r:
            r.run("3PCF", data, *mp, 32, 3500.0, b, assign="TSC", randoms=rand)
            d["zeta_" + tag] = r.zeta(*mp, b.n_rbin)
    np.savez_compressed(os.path.join(HERE, "survey_bk_zeta.npz"), **d)


def make_bk_256():
    """Box B_l on a 256^3 mesh with shells reaching |n| = 35 (4s + 1 = 141): the reduced
    chain grid is then 192 = 3 x 64, a non-power-of-two transform length.  From the numpy
    restatement (oracle/restate.py, pinned to the reference's outputs for TSC)."""
    from oracle import restate as R
    pos = lognormal_box(20000, 1000.0, ngrid=64, seed=19, exact_n=20000)
    b = Binning(0.03, 0.21, 7, 4.0, 156.0, 20)
    kb = R.bins(b.kmin, b.kmax, b.n_kbin)
    d = dict(pos=pos, boxsize=1000.0, n_mesh=256, binning=binning_arr(b))
    for mp in ((0, 0, 0), (2, 0, 2)):
        bk, sn, norm = R.bk_box(pos, 256, 1000.0, kb, *mp, R.TSC)
        d["bk_" + "".join(map(str, mp))] = norm * (bk - sn)
    np.savez_compressed(os.path.join(HERE, "box_bk_256.npz"), **d)


def make_extensions():
    """PCS assignment and interlacing are not in the reference: their fixtures come from
    the numpy restatement oracle/restate.py, which tests/test_oracle_restate.py pins to the
    reference's own outputs for NGP/CIC/TSC."""
    from oracle import restate as R
    pos = lognormal_box(15000, 1000.0, ngrid=32, seed=17, exact_n=15000)
    bp = Binning(0.005, 0.295, 30, 4.0, 156.0, 20)
    kb = R.bins(bp.kmin, bp.kmax, bp.n_kbin)
    d = dict(pos=pos, boxsize=1000.0, n_mesh=32, binning=binning_arr(bp))
    cases = (("PCS", False), ("PCS", True), ("TSC", True), ("CIC", True), ("NGP", True))
    for assign, il in cases:
        for ell in (0, 2, 4):
            pk, nm, norm = R.pk_box(pos, 32, 1000.0, kb, ell, R.SCHEMES[assign], interlace=il)
            d[f"pk_{assign}_{int(il)}_{ell}"] = norm * pk
            d[f"nmode_{assign}_{int(il)}"] = nm
    bb = Binning(0.015, 0.075, 7, 4.0, 156.0, 20)
    kb = R.bins(bb.kmin, bb.kmax, bb.n_kbin)
    d["bk_binning"] = binning_arr(bb)
    for assign, il in (("PCS", True), ("TSC", True), ("PCS", False)):
        for mp in ((0, 0, 0), (1, 1, 0), (2, 0, 2)):
            bk, sn, norm = R.bk_box(pos, 32, 1000.0, kb, *mp, R.SCHEMES[assign], interlace=il)
            d[f"bk_{assign}_{int(il)}_" + "".join(map(str, mp))] = norm * (bk - sn)
    np.savez_compressed(os.path.join(HERE, "box_extensions.npz"), **d)


def make_odd():
    """Multipoles with odd l1 + l2 (odd L): their shot-noise weights are odd in cos(theta),
    which exercises the histogram's sign handling, the Nyquist plane z = -L/2 included."""
    mps = ((1, 0, 1), (2, 1, 1))
    pos = lognormal_box(12000, 1000.0, ngrid=32, seed=12, exact_n=12000)
    bb = Binning(0.015, 0.075, 7, 4.0, 156.0, 20)
    d = dict(pos=pos, boxsize=1000.0, binning=binning_arr(bb), n_mesh=32)
    for mp, v in run_bk(pos, 32, 1000.0, bb, "TSC", mps=mps).items():
        d["bk_TSC_" + "".join(map(str, mp))] = v
    pz = lognormal_box(10000, 400.0, ngrid=32, seed=15, exact_n=10000)
    bz = Binning(0.02, 0.1, 5, 20.0, 140.0, 7)
    d["zeta_pos"] = pz
    d["zeta_boxsize"] = 400.0
    d["zeta_binning"] = binning_arr(bz)
    for mp, v in run_zeta(pz, 32, 400.0, bz, "TSC", mps=mps).items():
        d["zeta_TSC_" + "".join(map(str, mp))] = v
    np.savez_compressed(os.path.join(HERE, "box_odd.npz"), **d)


def make_xi():
    """Two-point correlation function multipoles: box (powerspec.hpp:334-393) for every
    scheme, survey (powerspec.hpp:93-180), window (powerspec.hpp:182-270) and the window
    3PCF (bispec.hpp:617-874), on the catalogues of the P and survey fixtures."""
    d = {}
    pos = lognormal_box(15000, 1000.0, ngrid=32, seed=11, exact_n=15000)
    bx = Binning(0.005, 0.295, 30, 4.0, 156.0, 20)
    d.update(box_pos=pos, box_binning=binning_arr(bx), box_boxsize=1000.0, box_n_mesh=64)
    for assign, ells in (("TSC", (0, 1, 2, 4)), ("CIC", (0, 2)), ("NGP", (0, 2))):
        for ell in ells:
            with ref_runner.RefRun() as r:
                r.run("2PCF", pos, ell, 0, ell, 64, 1000.0, bx, assign=assign)
                d[f"box_xi_{assign}_{ell}"] = r.xi(ell)[1]
    data, rand = survey_shell(3000, 60000, seed=16)
    bs = Binning(0.004, 0.048, 12, 100.0, 1500.0, 15)
    d.update(sv_data=data, sv_rand=rand, sv_binning=binning_arr(bs), sv_boxsize=3500.0, sv_n_mesh=64)
    for ell in (0, 1, 2):
        with ref_runner.RefRun() as r:
            r.run("2PCF", data, ell, 0, ell, 64, 3500.0, bs, assign="TSC", randoms=rand)
            d[f"sv_xi_{ell}"] = r.xi(ell)[1]
            sc = r.survey_scalars()
        with ref_runner.RefRun() as r:
            r.run("window2PCF", data, ell, 0, ell, 64, 3500.0, bs, assign="TSC", randoms=rand)
            d[f"win_xi_{ell}"] = r.xi(ell, window=True)[1]
    for k, v in sc.items():
        d[f"sv_scalars_{k}"] = v
    data3, rand3 = survey_shell(2000, 30000, seed=18)
    b3 = Binning(0.004, 0.02, 5, 150.0, 750.0, 5)
    d.update(w3_data=data3, w3_rand=rand3, w3_binning=binning_arr(b3), w3_boxsize=3500.0, w3_n_mesh=32)
    for mp in ((0, 0, 0), (1, 1, 0), (2, 0, 2)):
        with ref_runner.RefRun() as r:
            r.run("window3PCF", data3, *mp, 32, 3500.0, b3, assign="TSC", randoms=rand3)
            d["w3_zeta_" + "".join(map(str, mp))] = r.zeta_window(*mp, b3.n_rbin)
            sc = r.survey_scalars()
    for k, v in sc.items():
        d[f"w3_scalars_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "xi_window.npz"), **d)


def gadget_files(rng, n_per_file, time=0.5, box=1000.0):
    """Bytes of a Gadget-2 snapshot split over len(n_per_file) files (256-byte header, then
    position, velocity and id blocks, each between Fortran record markers)."""
    import struct
    total = sum(n_per_file)
    files, pos_all, vel_all = [], [], []
    for i, npf in enumerate(n_per_file):
        pos = rng.uniform(0.0, box, size=(npf, 3)).astype(np.float32)
        vel = rng.normal(0.0, 300.0, size=(npf, 3)).astype(np.float32)
        hdr = struct.pack("6I6dddii6Iii4d", 0, npf, 0, 0, 0, 0, 0.0, 1.5, 0, 0, 0, 0, time, 1.0 / time - 1.0, 0, 0,
                          0, total, 0, 0, 0, 0, 0, len(n_per_file), box, 0.31, 0.69, 0.68)
        hdr += b"\0" * (256 - len(hdr))
        rec = lambda b: struct.pack("i", len(b)) + b + struct.pack("i", len(b))
        ids = np.arange(npf, dtype=np.int64) + sum(n_per_file[:i])
        files.append(rec(hdr) + rec(pos.tobytes()) + rec(vel.tobytes()) + rec(ids.tobytes()))
        pos_all.append(pos)
        vel_all.append(vel)
    return files


def make_ingest():
    """The reference's own readers (readParticleBOSS particle.hpp:93-154,
    readParticlesFromGagdetSnapshot particleGadget.hpp:211-298) run through the harness on
    an ASCII file with lines that do and do not parse, and on a two-file Gadget snapshot."""
    import subprocess
    import tempfile
    rng = np.random.default_rng(23)
    lines = ["# x y z w", "", "1 2 3 4", "1 2 3", "1 2 3 4 5 6", "  5.5\t6.5  7.5 8.5\r", "1,2,3,4",
             "+1 -2 .3 4.", "1e5 2E-3 -0 0x1p3", "abc 1 2 3", "1 2 3 nan", "7 8 9 1e400", "\t", "3 4 5 6 # tail"]
    body = rng.uniform(-2000.0, 2000.0, size=(60000, 4))
    text = "\n".join(lines) + "\n" + "\n".join(" ".join(repr(float(v)) for v in row) for row in body) + "\n9 9 9 9"
    gfiles = gadget_files(rng, [3000, 2500])
    with tempfile.TemporaryDirectory() as tmp:
        ap = os.path.join(tmp, "cat.txt")
        with open(ap, "w") as f:
            f.write(text)
        gb = os.path.join(tmp, "snap")
        for i, b in enumerate(gfiles):
            with open(f"{gb}.{i}", "wb") as f:
                f.write(b)
        for mode, src in (("--read-ascii", ap), ("--read-gadget", gb)):
            subprocess.run([ref_runner.HARNESS, mode, src, os.path.join(tmp, mode + ".f64")], check=True)
        ascii_ref = np.fromfile(os.path.join(tmp, "--read-ascii.f64")).reshape(-1, 4)
        gadget_ref = np.fromfile(os.path.join(tmp, "--read-gadget.f64")).reshape(-1, 6)
    np.savez_compressed(os.path.join(HERE, "ingest.npz"), ascii_text=np.frombuffer(text.encode(), dtype=np.uint8),
                        ascii_ref=ascii_ref, gadget0=np.frombuffer(gfiles[0], dtype=np.uint8),
                        gadget1=np.frombuffer(gfiles[1], dtype=np.uint8), gadget_ref=gadget_ref)


def outside_catalogue(n_mesh: int, boxsize: float, n: int, seed: int) -> np.ndarray:
    """Particles partly outside the box: a quarter within 1.6 cells beyond a face (where the
    reference's int() truncation toward zero gives CIC/TSC weights above 1 for negative
    coordinates and the flat-index rule bleeds into neighbouring rows), and a few at up to
    three box lengths away on one axis (dropped, or landed elsewhere by the flat-index rule)."""
    rng = np.random.default_rng(seed)
    dr = boxsize / n_mesh
    pos = lognormal_box(n, boxsize, ngrid=n_mesh, seed=seed, exact_n=n)
    k = n // 4
    axis = rng.integers(0, 3, size=k)
    side = rng.random(k) < 0.5
    off = rng.uniform(0.0, 1.6 * dr, size=k)
    pos[np.arange(k), axis] = np.where(side, -off, boxsize + off)
    m = 40
    axis = rng.integers(0, 3, size=m)
    pos[k + np.arange(m), axis] = rng.uniform(-3.0 * boxsize, 4.0 * boxsize, size=m)
    return np.ascontiguousarray(pos)


def make_outside():
    """P_l and B_000 of a catalogue with particles outside the box (outside_catalogue), every
    assignment scheme of the reference: its bounds rule (field.hpp:92-96) applied to the
    anchors its int() truncation gives."""
    pos = outside_catalogue(32, 1000.0, 12000, seed=21)
    b = Binning(0.015, 0.095, 9, 4.0, 156.0, 20)  # below the 32^3 Nyquist k = 0.1
    d = dict(pos=pos, boxsize=1000.0, n_mesh=32, binning=binning_arr(b))
    for assign in ("NGP", "CIC", "TSC"):
        for ell, v in run_pk(pos, 32, 1000.0, b, assign, ells=(0, 2)).items():
            d[f"pk_{assign}_{ell}"] = v
        d[f"bk_{assign}_000"] = run_bk(pos, 32, 1000.0, b, assign, mps=((0, 0, 0),))[(0, 0, 0)]
    np.savez_compressed(os.path.join(HERE, "box_outside.npz"), **d)


def make_long_axes():
    """P_l on a [1024, 16, 1024] mesh: the longest line length the transforms support, on
    the strided (x) and the contiguous (z) axis."""
    pos = uniform_box(20000, 1000.0, seed=22)
    b = Binning(0.01, 0.15, 8, 4.0, 156.0, 20)
    nm = [1024, 16, 1024]
    d = dict(pos=pos, boxsize=np.array([1000.0, 1000.0, 1000.0]), n_mesh=np.array(nm), binning=binning_arr(b))
    for ell in (0, 2):
        with ref_runner.RefRun() as r:
            r.run("pk", pos, ell, 0, ell, nm, 1000.0, b)
            d[f"pk_{ell}"] = r.pk(ell)[1]
    np.savez_compressed(os.path.join(HERE, "box_long_axes.npz"), **d)


def make_mixed_meshes():
    """Meshes that are not powers of two, with unequal cell sizes (the reference transforms
    any n_mesh, e.g. its survey meshes 250 x 460 x 260): box P_l on a [60, 36, 50] mesh of a
    [1000, 800, 900] box; survey scalars and P_l on [50, 92, 52] (factors 2, 5, 23, 13);
    the survey reconstruction on a [30, 46, 26] mesh followed by P_l."""
    d = {}
    pos = lognormal_box(15000, 1000.0, ngrid=32, seed=23, exact_n=15000)
    pos = pos * np.array([1.0, 0.8, 0.9])
    bb = Binning(0.01, 0.13, 7, 4.0, 156.0, 20)
    nmb, bsb = [60, 36, 50], [1000.0, 800.0, 900.0]
    d.update(box_pos=pos, box_n_mesh=np.array(nmb), box_boxsize=np.array(bsb), box_binning=binning_arr(bb))
    for assign in ("TSC", "CIC"):
        for ell in (0, 2):
            with ref_runner.RefRun() as r:
                r.run("pk", pos, ell, 0, ell, nmb, bsb, bb, assign=assign)
                d[f"box_pk_{assign}_{ell}"] = r.pk(ell)[1]
    data, rand = survey_shell(3000, 60000, seed=24)
    bs = Binning(0.004, 0.048, 12, 20.0, 140.0, 7)
    nms = [50, 92, 52]
    d.update(sv_data=data, sv_rand=rand, sv_n_mesh=np.array(nms), sv_boxsize=3500.0, sv_binning=binning_arr(bs))
    for ell in (0, 2):
        with ref_runner.RefRun() as r:
            r.run("pk", data, ell, 0, ell, nms, 3500.0, bs, assign="TSC", randoms=rand)
            d[f"sv_pk_{ell}"] = r.pk(ell)[1]
            sc = r.survey_scalars()
    for k, v in sc.items():
        d[f"sv_scalars_{k}"] = v
    nrec = [30, 46, 26]
    d["sv_n_mesh_recon"] = np.array(nrec)
    with ref_runner.RefRun() as r:
        r.run("pk", data, 0, 0, 0, nms, 3500.0, bs, assign="TSC", randoms=rand, recon=(2.0, 40.0, nrec))
        a = ref_runner._read_cols(os.path.join(r.out, "pk0_recon.dat"))
        d["sv_recon_pk_0"] = a[:, 1] + 1j * a[:, 2]
        d["sv_recon_D"], d["sv_recon_R"] = r.recon_positions()
    np.savez_compressed(os.path.join(HERE, "mixed_meshes.npz"), **d)


def make_general_meshes():
    """The correlation-field statistics on meshes whose histograms take the general (octant
    key) path -- unequal cells, or a z axis that is not a power of two: box B and 2PCF on a
    [64, 36, 50] mesh of a [1000, 800, 900] box; box B and 3PCF on a cubic [48, 48, 48] mesh;
    survey B on [64, 92, 52] and the survey 2PCF on [50, 92, 52] (3500 Mpc/h cube)."""
    d = {}
    pos = lognormal_box(12000, 1000.0, ngrid=32, seed=25, exact_n=12000) * np.array([1.0, 0.8, 0.9])
    nmb, bsb = [64, 36, 50], [1000.0, 800.0, 900.0]
    bb = Binning(0.015, 0.075, 7, 20.0, 160.0, 8)
    d.update(box_pos=pos, box_n_mesh=np.array(nmb), box_boxsize=np.array(bsb), box_binning=binning_arr(bb))
    for mp in ((0, 0, 0), (2, 0, 2)):
        with ref_runner.RefRun() as r:
            r.run("bk", pos, *mp, nmb, bsb, bb, assign="TSC")
            d["box_bk_" + "".join(map(str, mp))] = r.bk(*mp, bb.n_kbin)
    for ell in (0, 2):
        with ref_runner.RefRun() as r:
            r.run("2PCF", pos, ell, 0, ell, nmb, bsb, bb, assign="TSC")
            d[f"box_xi_{ell}"] = r.xi(ell)[1]
    cub = lognormal_box(10000, 1000.0, ngrid=32, seed=26, exact_n=10000)
    bc = Binning(0.01, 0.04, 4, 20.0, 140.0, 7)
    d.update(cub_pos=cub, cub_n_mesh=48, cub_boxsize=1000.0, cub_binning=binning_arr(bc))
    with ref_runner.RefRun() as r:
        r.run("bk", cub, 2, 0, 2, 48, 1000.0, bc, assign="TSC")
        d["cub_bk_202"] = r.bk(2, 0, 2, bc.n_kbin)
    for mp in ((0, 0, 0), (1, 1, 0)):
        with ref_runner.RefRun() as r:
            r.run("3PCF", cub, *mp, 48, 1000.0, bc, assign="TSC")
            d["cub_zeta_" + "".join(map(str, mp))] = r.zeta(*mp, bc.n_rbin)
    for mp in ((0, 0, 0), (2, 0, 2)):  # the 3PCF on the non-cubic box (k-space octant keys)
        with ref_runner.RefRun() as r:
            r.run("3PCF", pos, *mp, nmb, bsb, bb, assign="TSC")
            d["box_zeta_" + "".join(map(str, mp))] = r.zeta(*mp, bb.n_rbin)
    data, rand = survey_shell(2000, 30000, seed=27)
    bs = Binning(0.004, 0.02, 5, 150.0, 750.0, 5)
    d.update(sv_data=data, sv_rand=rand, sv_boxsize=3500.0, sv_binning=binning_arr(bs),
             sv_bk_n_mesh=np.array([64, 92, 52]), sv_xi_n_mesh=np.array([50, 92, 52]))
    for mp in ((0, 0, 0), (2, 0, 2)):
        with ref_runner.RefRun() as r:
            r.run("bk", data, *mp, [64, 92, 52], 3500.0, bs, assign="TSC", randoms=rand)
            d["sv_bk_" + "".join(map(str, mp))] = r.bk(*mp, bs.n_kbin)
    for ell in (0, 2):
        with ref_runner.RefRun() as r:
            r.run("2PCF", data, ell, 0, ell, [50, 92, 52], 3500.0, bs, assign="TSC", randoms=rand)
            d[f"sv_xi_{ell}"] = r.xi(ell)[1]
    np.savez_compressed(os.path.join(HERE, "general_meshes.npz"), **d)


def make_recon():
    """BAO reconstruction (particle_reconstruction.hpp:12-402) through the reference's drivers:
    the shifted positions and the reconstructed P_l, survey (main.cpp:215-225, then
    calcPowerSpectrum with the _recon file name) and box (main_box.cpp:134-152, then
    calcPowerSpectrumForBOXForReconstruction, the bispectrum and the 3PCF)."""
    d = {}
    data, rand = survey_shell(3000, 60000, seed=16)
    bs = Binning(0.004, 0.048, 12, 100.0, 1500.0, 15)
    d.update(sv_data=data, sv_rand=rand, sv_binning=binning_arr(bs), sv_boxsize=3500.0, sv_n_mesh=64,
             sv_n_mesh_recon=32, sv_b1=2.0, sv_RG=40.0)
    for ell in (0, 2):
        with ref_runner.RefRun() as r:
            r.run("pk", data, ell, 0, ell, 64, 3500.0, bs, assign="TSC", randoms=rand, recon=(2.0, 40.0, 32))
            a = ref_runner._read_cols(os.path.join(r.out, f"pk{ell}_recon.dat"))
            d[f"sv_pk_{ell}"] = a[:, 1] + 1j * a[:, 2]
            d["sv_recon_D"], d["sv_recon_R"] = r.recon_positions()
            sc = r.survey_scalars()
    for k, v in sc.items():
        d[f"sv_scalars_{k}"] = v
    pos = lognormal_box(15000, 1000.0, ngrid=32, seed=11, exact_n=15000)
    rnd = uniform_box(30000, 1000.0, seed=31)
    bx = Binning(0.005, 0.295, 30, 4.0, 156.0, 20)
    d.update(box_pos=pos, box_rand=rnd, box_binning=binning_arr(bx), box_boxsize=1000.0, box_n_mesh=32,
             box_n_mesh_recon=32, box_b1=1.5, box_RG=20.0)
    for ell in (0, 2):
        with ref_runner.RefRun() as r:
            r.run("pk", pos, ell, 0, ell, 32, 1000.0, bx, assign="TSC", randoms=rnd, recon=(1.5, 20.0, 32),
                  box_recon=True, all_rows=False)
            a = ref_runner._read_cols(os.path.join(r.out, f"pk{ell}_recon.dat"))
            d[f"box_pk_{ell}"] = a[:, 1] + 1j * a[:, 2]
            d["box_recon_D"], d["box_recon_R"] = r.recon_positions()
    # reconstructed-box bispectrum and 3PCF (bispec.hpp:1426-1990): a coarser binning so
    # that the reference's per-row runs stay short
    bb = Binning(0.02, 0.08, 4, 20.0, 140.0, 7)
    d["box_bk_binning"] = binning_arr(bb)
    for mp in ((0, 0, 0), (2, 0, 2)):
        with ref_runner.RefRun() as r:
            r.run("bk", pos, *mp, 32, 1000.0, bb, assign="TSC", randoms=rnd, recon=(1.5, 20.0, 32), box_recon=True)
            d["box_bk_" + "".join(map(str, mp))] = r.bk(*mp, bb.n_kbin, tag="_recon")
    for mp in ((0, 0, 0), (1, 1, 0)):
        with ref_runner.RefRun() as r:
            r.run("3PCF", pos, *mp, 32, 1000.0, bb, assign="TSC", randoms=rnd, recon=(1.5, 20.0, 32),
                  box_recon=True)
            d["box_zeta_" + "".join(map(str, mp))] = r.zeta(*mp, bb.n_rbin, tag="_recon")
    np.savez_compressed(os.path.join(HERE, "recon.npz"), **d)


def catalogue_digest(pos: np.ndarray) -> np.ndarray:
    """Count, coordinate sums and sums of squares: the tests regenerate the large catalogues
    from their seeds and check these first, so a generator change cannot pass silently."""
    return np.array([pos.shape[0], *pos.sum(axis=0), *(pos * pos).sum(axis=0)], dtype=np.float64)


def make_config_sizes():
    """Reference outputs at the configurations' own sizes (the catalogues are regenerated
    from their seeds by the tests, so only outputs and a digest are stored):
      c1: 2x10^5 uniform particles (seed 1) in a 1000 Mpc/h box, 128^3 mesh, TSC, l = 0, 2, 4,
          kmin 0.005, kmax 0.295, 30 bins;
      c2: the clustered lognormal catalogue of 10^7 particles (256^3 Gaussian grid, seed 2),
          512^3 mesh, TSC, l = 0, 2, 4 on the bispectrum's 25 k bins 0.015-0.255, and the
          B_000 row ith_kbin = 0 against every k2 (bispec.hpp:877-1203 as one run does it).
    The 512^3 runs take minutes each on one core; they run concurrently."""
    from concurrent.futures import ThreadPoolExecutor
    pos1 = uniform_box(200_000, 1000.0, seed=1)
    b1 = Binning(0.005, 0.295, 30, 4.0, 156.0, 20)
    pos2 = lognormal_box(10_000_000, 1000.0, ngrid=256, seed=2, exact_n=10_000_000)
    b2 = Binning(0.015, 0.255, 25, 4.0, 156.0, 20)

    def pk_job(pos, nm, b, ell):
        with ref_runner.RefRun() as r:
            r.run("pk", pos, ell, 0, ell, nm, 1000.0, b, assign="TSC")
            return r.pk(ell)[1], r.wall

    def bk_job():
        with ref_runner.RefRun() as r:
            r.run("bk", pos2, 0, 0, 0, 512, 1000.0, b2, assign="TSC", all_rows=False, ith=0)
            a = ref_runner._read_cols(os.path.join(r.out, "bk000_00.dat"))
            return a[:, 2] + 1j * a[:, 3], r.wall

    d = dict(c1_digest=catalogue_digest(pos1), c1_binning=binning_arr(b1), c2_digest=catalogue_digest(pos2),
             c2_binning=binning_arr(b2))
    with ThreadPoolExecutor(max_workers=4) as ex:
        fb = ex.submit(bk_job)
        f2 = {ell: ex.submit(pk_job, pos2, 512, b2, ell) for ell in (0, 2, 4)}
        f1 = {ell: ex.submit(pk_job, pos1, 128, b1, ell) for ell in (0, 2, 4)}
        for ell in (0, 2, 4):
            d[f"c1_pk_{ell}"], d[f"c1_wall_{ell}"] = f1[ell].result()
            d[f"c2_pk_{ell}"], d[f"c2_wall_{ell}"] = f2[ell].result()
        d["c2_bk000_row0"], d["c2_bk_wall"] = fb.result()
    np.savez_compressed(os.path.join(HERE, "box_config_sizes.npz"), **d)


def main():
    if "--outside" in sys.argv or "--long" in sys.argv or "--mixed" in sys.argv or "--general" in sys.argv:
        if "--outside" in sys.argv:
            make_outside()
        if "--long" in sys.argv:
            make_long_axes()
        if "--mixed" in sys.argv:
            make_mixed_meshes()
        if "--general" in sys.argv:
            make_general_meshes()
        print("fixtures written")
        return
    if "--recon" in sys.argv:
        make_recon()
        print("fixtures written")
        return
    if "--ingest" in sys.argv:
        make_ingest()
        print("fixtures written")
        return
    if "--xi" in sys.argv:
        make_xi()
        print("fixtures written")
        return
    if "--configs" in sys.argv:
        make_config_sizes()
        print("fixtures written")
        return
    if "--extensions" in sys.argv or "--bk256" in sys.argv:
        if "--extensions" in sys.argv:
            make_extensions()
        if "--bk256" in sys.argv:
            make_bk_256()
        print("fixtures written")
        return
    if not ref_runner.available():
        raise SystemExit("build the oracle first: make -C oracle")
    if "--zeta" in sys.argv or "--survey" in sys.argv or "--survey3" in sys.argv or "--odd" in sys.argv:
        if "--zeta" in sys.argv:
            make_zeta()
        if "--odd" in sys.argv:
            make_odd()
        if "--survey" in sys.argv:
            make_survey()
        if "--survey3" in sys.argv:
            make_survey_three_point()
        print("fixtures written")
        return
    # smoke case
    pos = lognormal_box(20000, 1000.0, ngrid=32, seed=5, exact_n=20000)
    b = Binning(0.02, 0.08, 4, 4.0, 156.0, 20)
    pk = run_pk(pos, 32, 1000.0, b, "TSC", ells=(0,))
    bk = run_bk(pos, 32, 1000.0, b, "TSC", mps=((0, 0, 0),))
    np.savez_compressed(os.path.join(HERE, "smoke_box_32.npz"), pos=pos, n_mesh=32, boxsize=1000.0,
                        binning=binning_arr(b), pk0=pk[0], bk000=bk[(0, 0, 0)])

    # power spectrum multipoles, every assignment scheme, two meshes
    pos = lognormal_box(15000, 1000.0, ngrid=32, seed=11, exact_n=15000)
    bp = Binning(0.005, 0.295, 30, 4.0, 156.0, 20)
    d = dict(pos=pos, boxsize=1000.0, binning=binning_arr(bp))
    for nm in (32, 64):
        for assign in ("NGP", "CIC", "TSC"):
            for ell, v in run_pk(pos, nm, 1000.0, bp, assign).items():
                d[f"pk_{nm}_{assign}_{ell}"] = v
    np.savez_compressed(os.path.join(HERE, "box_pk.npz"), **d)

    # bispectrum multipoles, all rows, TSC; (000) also for NGP and CIC
    pos = lognormal_box(12000, 1000.0, ngrid=32, seed=12, exact_n=12000)
    bb = Binning(0.015, 0.075, 7, 4.0, 156.0, 20)
    d = dict(pos=pos, boxsize=1000.0, binning=binning_arr(bb), n_mesh=32)
    for mp, v in run_bk(pos, 32, 1000.0, bb, "TSC").items():
        d["bk_TSC_" + "".join(map(str, mp))] = v
    for assign in ("NGP", "CIC"):
        for mp, v in run_bk(pos, 32, 1000.0, bb, assign, mps=((0, 0, 0),)).items():
            d[f"bk_{assign}_" + "".join(map(str, mp))] = v
    np.savez_compressed(os.path.join(HERE, "box_bk.npz"), **d)

    # boundary-stress catalogue (flat-index bleed rule), P and B
    pos = edge_catalogue(16, 400.0, 6000, seed=13)
    be = Binning(0.02, 0.1, 5, 4.0, 156.0, 20)
    d = dict(pos=pos, boxsize=400.0, n_mesh=16, binning=binning_arr(be))
    for assign in ("NGP", "CIC", "TSC"):
        for ell, v in run_pk(pos, 16, 400.0, be, assign, ells=(0, 2)).items():
            d[f"pk_{assign}_{ell}"] = v
        d[f"bk_{assign}_000"] = run_bk(pos, 16, 400.0, be, assign, mps=((0, 0, 0),))[(0, 0, 0)]
    np.savez_compressed(os.path.join(HERE, "box_edges.npz"), **d)

    # a uniform catalogue on a non-cubic mesh (P only: shot-noise histograms need cubic cells)
    pos = uniform_box(8000, 1000.0, seed=14)
    bn = Binning(0.01, 0.15, 8, 4.0, 156.0, 20)
    d = dict(pos=pos, boxsize=np.array([1000.0, 1000.0, 1000.0]), n_mesh=np.array([16, 32, 64]),
             binning=binning_arr(bn))
    for ell in (0, 2):
        with ref_runner.RefRun() as r:
            r.run("pk", pos, ell, 0, ell, [16, 32, 64], 1000.0, bn)
            d[f"pk_{ell}"] = r.pk(ell)[1]
    np.savez_compressed(os.path.join(HERE, "box_noncubic.npz"), **d)
    make_zeta()
    make_survey()
    make_survey_three_point()
    make_extensions()
    make_bk_256()
    make_outside()
    make_long_axes()
    make_mixed_meshes()
    make_general_meshes()
    print("fixtures written")


if __name__ == "__main__":
    main()
