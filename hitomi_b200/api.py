"""Python host API over the C ABI (include/hitomi_gpu.h).

`Context` owns one hg_ctx (one GPU, one precision form).  Its methods return the
reference's raw FP64 sums (pk_save, bk_save, sn_save) as complex numpy arrays plus the
normalisation factor, so `norm * pk_save` is what the reference prints to pk{l}.dat
(src/hitomi_measurement/powerspec.hpp:316-327) and `norm * (bk_save - sn_save)` what it
prints to bk{l1}{l2}{L}_{ith}.dat (bispec.hpp:1184-1196).

Errors follow the reference's int-status convention at the ABI; here a non-zero status
raises HitomiError with the library's message.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

ASSIGN = {"NGP": _lib.HG_NGP, "CIC": _lib.HG_CIC, "TSC": _lib.HG_TSC, "PCS": _lib.HG_PCS}
PRECISION = {"fp64": _lib.HG_FP64, "fp32": _lib.HG_FP32}
# stages of the periodic-box pipeline an FP32 context can run in FP64 (hg_config.fp64_stages)
STAGES = {"density": _lib.HG_STAGE_DENSITY, "bk_signal": _lib.HG_STAGE_BK_SIGNAL, "bk_shot": _lib.HG_STAGE_BK_SHOT}


def stage_bits(stages) -> int:
    """A stage name list ("density", "bk_signal", "bk_shot") or an int bit set, as an int."""
    if isinstance(stages, int):
        return stages
    bits = 0
    for s in stages:
        if s not in STAGES:
            raise HitomiError(f"unknown FP64 stage {s!r}; expected one of {sorted(STAGES)}")
        bits |= STAGES[s]
    return bits


class HitomiError(RuntimeError):
    pass


class BatchError(HitomiError):
    """A batch stopped at a failing mock: `done` mocks completed, their results in `results`
    (the same dicts batch_run returns), so a caller resumes from mock `done`."""

    def __init__(self, msg, done, results):
        super().__init__(msg)
        self.done = done
        self.results = results


@dataclass
class Binning:
    kmin: float
    kmax: float
    n_kbin: int
    rmin: float = 30.0
    rmax: float = 150.0
    n_rbin: int = 25

    def kbin(self) -> np.ndarray:
        """ToolClass::setKbin (tools.hpp:118-124)."""
        dk = (self.kmax - self.kmin) / float(self.n_kbin - 1)
        return np.array([self.kmin + dk * float(i) for i in range(self.n_kbin)])

    def rbin(self) -> np.ndarray:
        """ToolClass::setRbin (tools.hpp:126-132)."""
        dr = (self.rmax - self.rmin) / float(self.n_rbin - 1)
        return np.array([self.rmin + dr * float(i) for i in range(self.n_rbin)])


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Context:
    def __init__(self, n_mesh, boxsize, binning: Binning, assign: str = "TSC", precision: str = "fp64",
                 periodic: bool = False, interlace: bool = False, device: int = 0, fp64_stages=(),
                 check_build: bool = False):
        """check_build: run on the check library (device-side bounds checks at the
        index-sensitive accesses; a failed check fails the call)."""
        self._lib = _lib.load(check=check_build)
        cfg = _lib.HgConfig()
        nm = [int(n_mesh)] * 3 if np.isscalar(n_mesh) else [int(v) for v in n_mesh]
        bs = [float(boxsize)] * 3 if np.isscalar(boxsize) else [float(v) for v in boxsize]
        for a in range(3):
            cfg.n_mesh[a] = nm[a]
            cfg.boxsize[a] = bs[a]
        if assign not in ASSIGN:
            raise HitomiError(f"assignment must be one of {sorted(ASSIGN)}")
        cfg.assign = ASSIGN[assign]
        cfg.interlace = int(bool(interlace))
        cfg.precision = PRECISION[precision]
        cfg.kmin, cfg.kmax, cfg.n_kbin = binning.kmin, binning.kmax, binning.n_kbin
        cfg.rmin, cfg.rmax, cfg.n_rbin = binning.rmin, binning.rmax, binning.n_rbin
        cfg.periodic = int(bool(periodic))
        cfg.device = int(device)
        cfg.fp64_stages = stage_bits(fp64_stages)
        self.n_mesh, self.boxsize, self.binning = nm, bs, binning
        self.precision = precision
        h = ctypes.c_void_p()
        if self._lib.hg_create(ctypes.byref(h), ctypes.byref(cfg)) != 0:
            raise HitomiError(self._lib.hg_last_error(None).decode())
        self._h = h
        self._keep = {}

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._lib.hg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise HitomiError(self._lib.hg_last_error(self._h).decode())

    # -- particles
    def set_particles(self, slot: int, arr: np.ndarray, pos_off: int = 0, los_off: int = -1, w_off: int = -1):
        """arr: (n, fields) float64 array of structs, C-contiguous (e.g. x y z or x y z vx vy vz)."""
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.ndim != 2:
            raise HitomiError("particle array must be 2-D (n, fields)")
        self._keep[slot] = a
        self._check(self._lib.hg_set_particles(self._h, slot, _dp(a), a.shape[0], a.shape[1] * 8, pos_off, los_off,
                                               w_off))

    def set_survey(self, data: np.ndarray, randoms: np.ndarray):
        """Data and randoms as (n, 7) {pos, los, w} records (hitomi_b200.survey.prepare)."""
        from . import survey
        for slot, arr in ((0, data), (1, randoms)):
            self.set_particles(slot, arr, pos_off=survey.POS_OFF, los_off=survey.LOS_OFF, w_off=survey.W_OFF)

    def set_particles_device(self, slot: int, ptr: int, n: int, stride_bytes: int, pos_off: int = 0,
                             los_off: int = -1, w_off: int = -1, keep=None):
        """Use a caller-owned device array (e.g. a torch CUDA tensor's data_ptr()) in place."""
        self._keep[slot] = keep
        self._check(self._lib.hg_set_particles_device(self._h, slot, ctypes.cast(ctypes.c_void_p(ptr),
                                                      ctypes.POINTER(ctypes.c_double)), n, stride_bytes, pos_off,
                                                      los_off, w_off))

    def set_profiling(self, on: bool = True):
        self._check(self._lib.hg_set_profiling(self._h, int(bool(on))))

    def kernel_stats(self) -> dict:
        buf = ctypes.create_string_buffer(1 << 16)
        self._check(self._lib.hg_kernel_stats(self._h, buf, len(buf)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms, by = line.split("\t")
            out[name] = dict(launches=int(n), ms=float(ms), bytes=float(by))
        return out

    def set_memory_limit(self, nbytes: int):
        """Cap the device memory this context's buffers may hold (0: no cap)."""
        self._check(self._lib.hg_set_memory_limit(self._h, int(nbytes)))

    def memory_in_use(self) -> int:
        """Bytes of device memory the context's buffers hold now."""
        return int(self._lib.hg_memory_in_use(self._h))

    def tuning(self) -> str:
        """The launch shapes the context's autotuner picked, with the time of every variant."""
        buf = ctypes.create_string_buffer(1 << 14)
        self._check(self._lib.hg_tuning(self._h, buf, len(buf)))
        return buf.value.decode()

    # -- statistics
    def pk_box(self, ell: int):
        nk = self.binning.n_kbin
        out = np.zeros(2 * nk)
        nmode = np.zeros(nk, dtype=np.int32)
        norm = ctypes.c_double()
        self._check(self._lib.hg_pk_box(self._h, ell, _dp(out), nmode.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                        ctypes.byref(norm)))
        return out[0::2] + 1j * out[1::2], nmode, norm.value

    def bk_box(self, ell1: int, ell2: int, ELL: int, ith_kbin: int = -1):
        nk = self.binning.n_kbin
        rows = nk if ith_kbin < 0 else 1
        bk = np.zeros(2 * rows * nk)
        sn = np.zeros(2 * rows * nk)
        norm = ctypes.c_double()
        self._check(self._lib.hg_bk_box(self._h, ell1, ell2, ELL, ith_kbin, _dp(bk), _dp(sn), ctypes.byref(norm)))
        c = lambda v: (v[0::2] + 1j * v[1::2]).reshape(rows, nk)
        return c(bk), c(sn), norm.value

    def bk_box_multi(self, multipoles, ith_kbin: int = -1):
        """Several (ell1, ell2, ELL) multipoles at once; returns lists of (bk, sn) and norm."""
        nk = self.binning.n_kbin
        rows = nk if ith_kbin < 0 else 1
        m = len(multipoles)
        ells = np.array([v for mp in multipoles for v in mp], dtype=np.int32)
        bk = np.zeros(2 * m * rows * nk)
        sn = np.zeros(2 * m * rows * nk)
        norm = ctypes.c_double()
        self._check(self._lib.hg_bk_box_multi(self._h, m, ells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                              ith_kbin, _dp(bk), _dp(sn), ctypes.byref(norm)))
        c = lambda v: (v[0::2] + 1j * v[1::2]).reshape(m, rows, nk)
        return c(bk), c(sn), norm.value

    def zeta_box(self, ell1: int, ell2: int, ELL: int, ith_rbin: int = -1):
        nr = self.binning.n_rbin
        rows = nr if ith_rbin < 0 else 1
        z = np.zeros(2 * rows * nr)
        sn = np.zeros(2 * rows * nr)
        norm = ctypes.c_double()
        self._check(self._lib.hg_zeta_box(self._h, ell1, ell2, ELL, ith_rbin, _dp(z), _dp(sn), ctypes.byref(norm)))
        c = lambda v: (v[0::2] + 1j * v[1::2]).reshape(rows, nr)
        return c(z), c(sn), norm.value

    def zeta_box_multi(self, multipoles, ith_rbin: int = -1):
        """Several (ell1, ell2, ELL) 3PCF multipoles at once: arrays [m][rows][n_rbin] and norm."""
        nr = self.binning.n_rbin
        rows = nr if ith_rbin < 0 else 1
        m = len(multipoles)
        ells = np.array([v for mp in multipoles for v in mp], dtype=np.int32)
        z = np.zeros(2 * m * rows * nr)
        sn = np.zeros(2 * m * rows * nr)
        norm = ctypes.c_double()
        self._check(self._lib.hg_zeta_box_multi(self._h, m, ells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                ith_rbin, _dp(z), _dp(sn), ctypes.byref(norm)))
        c = lambda v: (v[0::2] + 1j * v[1::2]).reshape(m, rows, nr)
        return c(z), c(sn), norm.value

    def _survey_three_point(self, fn, nbins, multipoles, ith, alpha, vsurvey):
        rows = nbins if ith < 0 else 1
        m = len(multipoles)
        ells = np.array([v for mp in multipoles for v in mp], dtype=np.int32)
        a = np.zeros(2 * m * rows * nbins)
        sn = np.zeros(2 * m * rows * nbins)
        norm = ctypes.c_double()
        self._check(fn(self._h, m, ells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ith, float(alpha),
                       float(vsurvey), _dp(a), _dp(sn), ctypes.byref(norm)))
        c = lambda v: (v[0::2] + 1j * v[1::2]).reshape(m, rows, nbins)
        return c(a), c(sn), norm.value

    def bk_survey_multi(self, multipoles, alpha: float, vsurvey: float, ith_kbin: int = -1):
        """Survey bispectrum multipoles: arrays [m][rows][n_kbin] and norm."""
        return self._survey_three_point(self._lib.hg_bk_survey_multi, self.binning.n_kbin, multipoles, ith_kbin,
                                        alpha, vsurvey)

    def bk_survey(self, ell1: int, ell2: int, ELL: int, alpha: float, vsurvey: float, ith_kbin: int = -1):
        bk, sn, norm = self.bk_survey_multi(((ell1, ell2, ELL),), alpha, vsurvey, ith_kbin)
        return bk[0], sn[0], norm

    def zeta_survey_multi(self, multipoles, alpha: float, vsurvey: float, ith_rbin: int = -1):
        """Survey 3PCF multipoles: arrays [m][rows][n_rbin] and norm."""
        return self._survey_three_point(self._lib.hg_zeta_survey_multi, self.binning.n_rbin, multipoles, ith_rbin,
                                        alpha, vsurvey)

    def zeta_survey(self, ell1: int, ell2: int, ELL: int, alpha: float, vsurvey: float, ith_rbin: int = -1):
        z, sn, norm = self.zeta_survey_multi(((ell1, ell2, ELL),), alpha, vsurvey, ith_rbin)
        return z[0], sn[0], norm

    def survey_scalars(self):
        vals = [ctypes.c_double() for _ in range(5)]
        self._check(self._lib.hg_survey_scalars(self._h, *[ctypes.byref(v) for v in vals]))
        return tuple(v.value for v in vals)

    def pk_survey(self, ell: int, alpha: float, vsurvey: float):
        nk = self.binning.n_kbin
        out = np.zeros(2 * nk)
        nmode = np.zeros(nk, dtype=np.int32)
        norm = ctypes.c_double()
        self._check(self._lib.hg_pk_survey(self._h, ell, alpha, vsurvey, _dp(out),
                                           nmode.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(norm)))
        return out[0::2] + 1j * out[1::2], nmode, norm.value

    def _xi(self, fn, *args):
        nr = self.binning.n_rbin
        out = np.zeros(2 * nr)
        nmode = np.zeros(nr, dtype=np.int32)
        norm = ctypes.c_double()
        self._check(fn(self._h, *args, _dp(out), nmode.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                       ctypes.byref(norm)))
        return out[0::2] + 1j * out[1::2], nmode, norm.value

    def xi_box(self, ell: int):
        """2PCF multipole of the box: (xi_save, cells per r bin, norm); the file value is
        norm * xi_save.real (powerspec.hpp:334-393)."""
        return self._xi(self._lib.hg_xi_box, int(ell))

    def xi_survey(self, ell: int, alpha: float, vsurvey: float):
        return self._xi(self._lib.hg_xi_survey, int(ell), float(alpha), float(vsurvey))

    def xi_window(self, ell: int, vsurvey: float):
        return self._xi(self._lib.hg_xi_window, int(ell), float(vsurvey))

    def _one_scalar_three_point(self, fn, nbins, multipoles, ith, scalar):
        rows = nbins if ith < 0 else 1
        m = len(multipoles)
        ells = np.array([v for mp in multipoles for v in mp], dtype=np.int32)
        z = np.zeros(2 * m * rows * nbins)
        sn = np.zeros(2 * m * rows * nbins)
        norm = ctypes.c_double()
        self._check(fn(self._h, m, ells.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ith, float(scalar), _dp(z),
                       _dp(sn), ctypes.byref(norm)))
        c = lambda v: (v[0::2] + 1j * v[1::2]).reshape(m, rows, nbins)
        return c(z), c(sn), norm.value

    def zeta_window_multi(self, multipoles, vsurvey: float, ith_rbin: int = -1):
        """Window 3PCF multipoles of the randoms (slot 1): arrays [m][rows][n_rbin] and norm."""
        return self._one_scalar_three_point(self._lib.hg_zeta_window_multi, self.binning.n_rbin, multipoles,
                                            ith_rbin, vsurvey)

    def bk_box_recon_multi(self, multipoles, alpha: float, ith_kbin: int = -1):
        """Reconstructed-box bispectrum multipoles of data (slot 0) and randoms (slot 1):
        arrays [m][rows][n_kbin] and norm (V^2 / N_D^3)."""
        return self._one_scalar_three_point(self._lib.hg_bk_box_recon_multi, self.binning.n_kbin, multipoles,
                                            ith_kbin, alpha)

    def zeta_box_recon_multi(self, multipoles, alpha: float, ith_rbin: int = -1):
        """Reconstructed-box 3PCF multipoles: arrays [m][rows][n_rbin] and norm (V^2 / N_D^3)."""
        return self._one_scalar_three_point(self._lib.hg_zeta_box_recon_multi, self.binning.n_rbin, multipoles,
                                            ith_rbin, alpha)

    def reconstruct(self, b1_fid: float, RG: float, box: bool = False, alpha: float = 0.0, vsurvey: float = 0.0):
        """BAO reconstruction of the current data (slot 0) and randoms (slot 1): their shifted
        positions as two (n, 3) arrays (particle_reconstruction.hpp:12-402)."""
        nd = self._keep[0].shape[0]
        nr = self._keep[1].shape[0]
        pd, pr = np.zeros((nd, 3)), np.zeros((nr, 3))
        self._check(self._lib.hg_reconstruct(self._h, int(bool(box)), float(b1_fid), float(RG), float(alpha),
                                             float(vsurvey), _dp(pd), _dp(pr)))
        return pd, pr

    def pk_box_recon(self, ell: int, alpha: float):
        nk = self.binning.n_kbin
        out = np.zeros(2 * nk)
        nmode = np.zeros(nk, dtype=np.int32)
        norm = ctypes.c_double()
        self._check(self._lib.hg_pk_box_recon(self._h, int(ell), float(alpha), _dp(out),
                                              nmode.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(norm)))
        return out[0::2] + 1j * out[1::2], nmode, norm.value

    def xi_box_recon(self, ell: int, alpha: float):
        return self._xi(self._lib.hg_xi_box_recon, int(ell), float(alpha))

    def batch_run(self, mocks, pk_ells=(), bk_multipoles=(), zeta_multipoles=()):
        """Box statistics of several catalogues through hg_batch_run (the next catalogue is
        copied to the GPU while the current one is measured).  mocks: (n, fields) float64
        arrays of structs with x y z first.  Returns one dict per mock: "pk" [n_pk][n_kbin],
        "pk_norm" [n_pk], "bk", "bk_sn" [n_bk][n_kbin][n_kbin], "bk_norm", "zeta", "zeta_sn"
        [n_zeta][n_rbin][n_rbin], "zeta_norm" (complex raw sums and their norms)."""
        arrs = [np.ascontiguousarray(m, dtype=np.float64) for m in mocks]
        ms = (_lib.HgMock * len(arrs))()
        for i, a in enumerate(arrs):
            ms[i].base = _dp(a)
            ms[i].n = a.shape[0]
            ms[i].stride_bytes = a.shape[1] * 8
            ms[i].pos_off = 0
        pk = np.array(list(pk_ells), dtype=np.int32)
        bk = np.array([v for mp in bk_multipoles for v in mp], dtype=np.int32)
        zt = np.array([v for mp in zeta_multipoles for v in mp], dtype=np.int32)
        npk, nbk, nz = len(pk), len(bk) // 3, len(zt) // 3
        blk = int(self._lib.hg_batch_block_len(self._h, npk, nbk, nz))
        out = np.zeros(blk * len(arrs))
        ip = lambda v: v.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        rc = self._lib.hg_batch_run(self._h, ms, len(arrs), npk, ip(pk), nbk, ip(bk), nz, ip(zt), _dp(out))
        done = len(arrs) if rc == 0 else int(self._lib.hg_batch_done(self._h))
        nk, nr = self.binning.n_kbin, self.binning.n_rbin
        res = []
        for i in range(done):
            o = out[i * blk:(i + 1) * blk]
            r, p = {}, 0
            c = lambda v, *shape: (v[0::2] + 1j * v[1::2]).reshape(shape)
            r["pk"] = c(o[p:p + 2 * npk * nk], npk, nk)
            p += 2 * npk * nk
            r["pk_norm"] = o[p:p + npk].copy()
            p += npk
            if nbk:
                sz = 2 * nbk * nk * nk
                r["bk"], r["bk_sn"] = c(o[p:p + sz], nbk, nk, nk), c(o[p + sz:p + 2 * sz], nbk, nk, nk)
                r["bk_norm"] = float(o[p + 2 * sz])
                p += 2 * sz + 1
            if nz:
                sz = 2 * nz * nr * nr
                r["zeta"], r["zeta_sn"] = c(o[p:p + sz], nz, nr, nr), c(o[p + sz:p + 2 * sz], nz, nr, nr)
                r["zeta_norm"] = float(o[p + 2 * sz])
            res.append(r)
        if rc != 0:
            raise BatchError(self._lib.hg_last_error(self._h).decode(), done, res)
        return res

    def last_timing(self):
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        self._lib.hg_last_timing(self._h, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value
