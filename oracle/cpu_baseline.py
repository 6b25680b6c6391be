"""TEST / BENCH INFRASTRUCTURE ONLY: the reference's CPU cost of one mock of the
periodic-box P_l + B_l workload, from a bounded sample.

The reference computes one k1 row of one bispectrum multipole per process run
(src/hitomi_measurement/main.cpp:78-84, bispec.hpp:877-1203) and one P_l per run
(powerspec.hpp:273-332).  A full 512^3 mock is hours of CPU, so it is not run end to
end.  Instead each building block the reference's drivers call is timed once at the
full mesh and particle count (oracle/_ref/ref_harness --unit OP, one single-threaded
process per block, run concurrently), and the per-mock time is the sum over the
reference's control flow of (number of calls) x (unit time):

  P_l (one run per l)         assign + fft + bin_l
  B row, multipole with C (m1, m2) terms (bispec.hpp:909-1182):
    shot noise, part 1        2 (assign + fft) + sum_terms [(l2 == 0) + (l1 == 0)] bin
    shot noise, part 2        2 (assign + fft) + 2 spline + C (2 ylmx + xi_ijk + nk snloop)
    signal                    2 (assign + fft) + corr + ifft + C (2 ylmk + shell + nk (shell + triple))
  mock = sum_l P_l + sum_multipoles nk rows.

Throughput follows the reference's own parallel pattern, one independent single-core
process per realization (main.cpp:64-76): mocks/s = cores / (per-mock seconds).
"""
from __future__ import annotations

import os
import subprocess
import tempfile
import shutil
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import ref_runner

UNIT_OPS = ("assign", "fft", "ifft", "corr", "bin_l0", "bin_l2", "xi_ijk", "ylmk", "ylmx", "shell", "triple",
            "snloop", "spline")


def _w3j_terms(l1, l2, L):
    """(m1, m2) pairs with M = 0 and |w| >= 1e-10 (bispec.hpp:923-931)."""
    from math import sqrt  # noqa: F401
    terms = []
    try:
        from sympy.physics.wigner import wigner_3j
    except Exception:  # pragma: no cover
        wigner_3j = None
    for m1 in range(-l1, l1 + 1):
        for m2 in range(-l2, l2 + 1):
            if m1 + m2 != 0:
                continue
            if wigner_3j is not None:
                w = float(wigner_3j(l1, l2, L, 0, 0, 0) * wigner_3j(l1, l2, L, m1, m2, 0))
                w *= (2 * L + 1) * (2 * l1 + 1) * (2 * l2 + 1)
                if abs(w) < 1e-10:
                    continue
            terms.append((m1, m2))
    return terms


def per_mock_seconds(unit: dict, nk: int, pk_ells=(0, 2, 4), multipoles=((0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2))):
    af = unit["assign"] + unit["fft"]
    t = 0.0
    for ell in pk_ells:
        t += af + (unit["bin_l0"] if ell == 0 else unit["bin_l2"])
    for (l1, l2, L) in multipoles:
        terms = _w3j_terms(l1, l2, L)
        C = len(terms)
        row = 0.0
        row += 2 * af + sum(((l2 == 0) + (l1 == 0)) * (unit["bin_l0"] if (l1 == 0 and l2 == 0) else unit["bin_l2"])
                            for _ in terms)
        row += 2 * af + 2 * unit["spline"] + C * (2 * unit["ylmx"] + unit["xi_ijk"] + nk * unit["snloop"])
        row += 2 * af + unit["corr"] + unit["ifft"] + C * (2 * unit["ylmk"] + unit["shell"] +
                                                           nk * (unit["shell"] + unit["triple"]))
        t += nk * row
    return t


def measure_units(pos: np.ndarray, n_mesh: int, boxsize: float, binning, ops=UNIT_OPS, concurrent: bool = True,
                  timeout: float = 600.0) -> dict:
    """Run each unit op once in its own process; returns {op: seconds}."""
    if not ref_runner.available():
        raise RuntimeError("oracle/_ref/ref_harness is not built")
    d = tempfile.mkdtemp(prefix="hxunit_")
    try:
        param = os.path.join(d, "param.ini")
        ref_runner.write_param(param, os.path.join(d, "out"), "bk", 0, 0, 0, n_mesh, boxsize, binning.kmin,
                               binning.kmax, binning.n_kbin, binning.rmin, binning.rmax, binning.n_rbin, "TSC")
        # the concurrent processes share one output directory: made here, since each would
        # otherwise race to create it (parameter.hpp:256-275 fails when mkdir loses)
        os.makedirs(os.path.join(d, "out"), exist_ok=True)
        dpath = os.path.join(d, "data.f64")
        np.ascontiguousarray(pos, dtype=np.float64).tofile(dpath)

        def one(op):
            p = subprocess.run([ref_runner.HARNESS, param, dpath, "--unit", op], capture_output=True, text=True,
                               timeout=timeout)
            if p.returncode != 0:
                raise RuntimeError(f"unit {op} failed: {p.stderr[-500:]}")
            for line in p.stdout.splitlines():
                if line.startswith("HX_UNIT"):
                    _, name, sec = line.split()
                    return name, float(sec)
            raise RuntimeError(f"unit {op}: no timing line")

        workers = len(ops) if concurrent else 1
        with ThreadPoolExecutor(max_workers=workers) as ex:
            res = dict(ex.map(one, ops))
        return res
    finally:
        shutil.rmtree(d, ignore_errors=True)


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def baseline(pos, n_mesh, boxsize, binning, pk_ells=(0, 2, 4),
             multipoles=((0, 0, 0), (1, 1, 0), (2, 0, 2), (0, 2, 2)), concurrent=True):
    t0 = time.perf_counter()
    unit = measure_units(pos, n_mesh, boxsize, binning, concurrent=concurrent)
    wall = time.perf_counter() - t0
    sec = per_mock_seconds(unit, binning.n_kbin, pk_ells, multipoles)
    cores = host_cores()
    return dict(mocks_per_s=cores / sec, per_mock_seconds=sec, cores=cores, unit_seconds=unit,
                sample_wall_seconds=wall)
