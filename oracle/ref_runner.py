"""TEST INFRASTRUCTURE ONLY: drive oracle/_ref/ref_harness (the reference's own estimator
headers compiled against the project-written FFTW/GSL shims, oracle/Makefile).

Writes a parameter file in the reference's format (every key its checkParameters
validates, src/hitomi_measurement/parameter.hpp:389-621), the particle arrays as raw
float64, runs the harness with full-precision output, and parses the result files the
reference writes (pk{l}.dat powerspec.hpp:319-327, bk{l1}{l2}{L}_{ith}.dat
bispec.hpp:1187-1196, zeta{l1}{l2}{L}_{ith}.dat bispec.hpp:1408-1416).
Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this module.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "ref_harness")


def available() -> bool:
    return os.path.exists(HARNESS) and os.access(HARNESS, os.X_OK)


def write_param(path: str, out_dir: str, measure: str, ell1: int, ell2: int, ELL: int, n_mesh, boxsize,
                kmin: float, kmax: float, n_kbin: int, rmin: float, rmax: float, n_rbin: int, assign: str = "TSC",
                ith_kbin: int = 0, ith_rbin: int = 0, recon=None):
    """recon: None, or (b1_fid, RG, n_mesh_recon) for flag_recon = True."""
    nm = [n_mesh] * 3 if np.isscalar(n_mesh) else list(n_mesh)
    b1, rg, nrec = (1.0, 15.0, nm) if recon is None else (recon[0], recon[1], recon[2])
    nrec = [nrec] * 3 if np.isscalar(nrec) else list(nrec)
    bs = [boxsize] * 3 if np.isscalar(boxsize) else list(boxsize)
    lines = [
        f"data_dir = {os.path.dirname(out_dir)}",
        "data_file = data.f64",
        "random_file = random.f64",
        f"output_dir = {out_dir}",
        f"measure = {measure}",
        "realization = 0",
        f"ell1 = {ell1}",
        f"ell2 = {ell2}",
        f"ELL = {ELL}",
        f"boxsize_x = {bs[0]!r}",
        f"boxsize_y = {bs[1]!r}",
        f"boxsize_z = {bs[2]!r}",
        f"n_mesh_x = {nm[0]}",
        f"n_mesh_y = {nm[1]}",
        f"n_mesh_z = {nm[2]}",
        f"kmin = {kmin!r}",
        f"kmax = {kmax!r}",
        f"n_kbin = {n_kbin}",
        f"rmin = {rmin!r}",
        f"rmax = {rmax!r}",
        f"n_rbin = {n_rbin}",
        f"flag_recon = {'False' if recon is None else 'True'}",
        f"b1_fid = {b1!r}",
        f"RG = {rg!r}",
        f"n_mesh_recon_x = {nrec[0]}",
        f"n_mesh_recon_y = {nrec[1]}",
        f"n_mesh_recon_z = {nrec[2]}",
        f"ith_kbin = {ith_kbin}",
        f"ith_rbin = {ith_rbin}",
        "NR = 0",
        "data_mpi_file = none",
        "sim_data = Gadget",
        "flag_RSD = False",
        "log10_Mmin = 12.9",
        "log10_Mmax = 13.5",
        f"assignment = {assign}",
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _read_cols(path: str) -> np.ndarray:
    return np.loadtxt(path, comments="#", ndmin=2)


class RefRun:
    """One harness invocation in a temporary directory."""

    def __init__(self, keep: bool = False):
        if not available():
            raise RuntimeError("oracle/_ref/ref_harness is not built (make -C oracle)")
        self.dir = tempfile.mkdtemp(prefix="hxref_")
        self.out = os.path.join(self.dir, "out")
        self.keep = keep
        self.wall = None

    def close(self):
        if not self.keep:
            shutil.rmtree(self.dir, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, measure: str, data: np.ndarray, ell1: int, ell2: int, ELL: int, n_mesh, boxsize, binning,
            assign: str = "TSC", randoms: np.ndarray | None = None, all_rows: bool = True, ith: int = 0,
            full: bool = True, timeout: float | None = None, recon=None, box_recon: bool = False):
        param = os.path.join(self.dir, "param.ini")
        write_param(param, self.out, measure, ell1, ell2, ELL, n_mesh, boxsize, binning.kmin, binning.kmax,
                    binning.n_kbin, binning.rmin, binning.rmax, binning.n_rbin, assign,
                    ith_kbin=ith, ith_rbin=ith, recon=recon)
        dpath = os.path.join(self.dir, "data.f64")
        np.ascontiguousarray(data, dtype=np.float64).tofile(dpath)
        args = [HARNESS, param, dpath]
        if randoms is not None:
            rpath = os.path.join(self.dir, "random.f64")
            np.ascontiguousarray(randoms, dtype=np.float64).tofile(rpath)
            args.append(rpath)
        if all_rows:
            args.append("--all-rows")
        if box_recon:
            args.append("--box-recon")
        env = dict(os.environ)
        if full:
            env["HX_FULL"] = "1"
        env["HX_TIMING"] = "1"
        t0 = time.perf_counter()
        p = subprocess.run(args, env=env, capture_output=True, text=True, timeout=timeout)
        self.wall_outer = time.perf_counter() - t0
        if p.returncode != 0:
            raise RuntimeError(f"ref_harness failed ({p.returncode}): {p.stderr[-2000:]}")
        for line in p.stdout.splitlines():
            if line.startswith("HX_WALL_SECONDS"):
                self.wall = float(line.split()[1])
        return self

    # ---- result readers
    def pk(self, ell: int):
        a = _read_cols(os.path.join(self.out, f"pk{ell}.dat"))
        return a[:, 0], a[:, 1] + 1j * a[:, 2]

    def bk(self, l1: int, l2: int, L: int, n_rows: int, tag: str = ""):
        rows = []
        for i in range(n_rows):
            a = _read_cols(os.path.join(self.out, f"bk{l1}{l2}{L}_{i:02d}{tag}.dat"))
            rows.append(a[:, 2] + 1j * a[:, 3])
        return np.array(rows)

    def zeta(self, l1: int, l2: int, L: int, n_rows: int, tag: str = ""):
        rows = []
        for i in range(n_rows):
            a = _read_cols(os.path.join(self.out, f"zeta{l1}{l2}{L}_{i:02d}{tag}.dat"))
            rows.append(a[:, 2])
        return np.array(rows)

    def xi(self, ell: int, window: bool = False):
        """xi{l}.dat / xi{l}_window.dat (powerspec.hpp:165-175, 254-264, 380-387): r, value."""
        a = _read_cols(os.path.join(self.out, f"xi{ell}{'_window' if window else ''}.dat"))
        return a[:, 0], a[:, 1]

    def zeta_window(self, l1: int, l2: int, L: int, n_rows: int):
        """zeta{l1}{l2}{L}_{ith}_window.dat (bispec.hpp:857-866)."""
        rows = []
        for i in range(n_rows):
            a = _read_cols(os.path.join(self.out, f"zeta{l1}{l2}{L}_{i:02d}_window.dat"))
            rows.append(a[:, 2])
        return np.array(rows)

    def recon_positions(self):
        """The reconstructed positions the harness wrote (recon_D.f64, recon_R.f64): (n, 3) each."""
        return tuple(np.fromfile(os.path.join(self.out, f"recon_{s}.f64")).reshape(-1, 3) for s in "DR")

    def survey_scalars(self):
        v = np.loadtxt(os.path.join(self.out, "survey_scalars_full"))
        return dict(alpha=v[0], vsurvey=v[1], nbar=v[2], wsum_data=v[3], wsum_rand=v[4])

    def text(self, name: str) -> str:
        with open(os.path.join(self.out, name)) as f:
            return f.read()
