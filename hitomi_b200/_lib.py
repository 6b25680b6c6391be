"""ctypes binding of the C ABI in include/hitomi_gpu.h.

The shared library is built in-tree (hitomi_b200/build.py).  There is no fallback:
if the library is missing or a GPU call fails, the error surfaces to the caller.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhitomi_b200.so")

# exported symbols, in include/hitomi_gpu.h order
SYMBOLS = (
    "hg_create",
    "hg_destroy",
    "hg_last_error",
    "hg_set_particles",
    "hg_set_particles_device",
    "hg_pk_box",
    "hg_bk_box",
    "hg_bk_box_multi",
    "hg_zeta_box",
    "hg_zeta_box_multi",
    "hg_bk_survey",
    "hg_bk_survey_multi",
    "hg_zeta_survey",
    "hg_zeta_survey_multi",
    "hg_survey_scalars",
    "hg_pk_survey",
    "hg_xi_box",
    "hg_xi_survey",
    "hg_xi_window",
    "hg_zeta_window",
    "hg_zeta_window_multi",
    "hg_reconstruct",
    "hg_pk_box_recon",
    "hg_xi_box_recon",
    "hg_bk_box_recon_multi",
    "hg_zeta_box_recon_multi",
    "hg_batch_run",
    "hg_batch_block_len",
    "hg_batch_done",
    "hg_set_memory_limit",
    "hg_memory_in_use",
    "hg_read_ascii",
    "hg_read_gadget",
    "hg_free",
    "hg_set_profiling",
    "hg_kernel_stats",
    "hg_tuning",
    "hg_pk_box_spectrum_static",
    "hg_last_timing",
)

HG_NGP, HG_CIC, HG_TSC, HG_PCS = 0, 1, 2, 3
HG_FP64, HG_FP32 = 0, 1
HG_STAGE_DENSITY, HG_STAGE_BK_SIGNAL, HG_STAGE_BK_SHOT = 1, 2, 4


class HgMock(ctypes.Structure):
    _fields_ = [
        ("base", ctypes.POINTER(ctypes.c_double)),
        ("n", ctypes.c_longlong),
        ("stride_bytes", ctypes.c_longlong),
        ("pos_off", ctypes.c_int),
    ]


class HgGadgetHeader(ctypes.Structure):
    _fields_ = [
        ("npart", ctypes.c_uint * 6),
        ("mass", ctypes.c_double * 6),
        ("time", ctypes.c_double),
        ("redshift", ctypes.c_double),
        ("flag_sfr", ctypes.c_int),
        ("flag_feedback", ctypes.c_int),
        ("npartTotal", ctypes.c_uint * 6),
        ("flag_cooling", ctypes.c_int),
        ("num_files", ctypes.c_int),
        ("BoxSize", ctypes.c_double),
        ("Omega0", ctypes.c_double),
        ("OmegaLambda", ctypes.c_double),
        ("HubbleParam", ctypes.c_double),
        ("fill", ctypes.c_char * 96),
    ]


class HgConfig(ctypes.Structure):
    _fields_ = [
        ("n_mesh", ctypes.c_int * 3),
        ("boxsize", ctypes.c_double * 3),
        ("assign", ctypes.c_int),
        ("interlace", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("kmin", ctypes.c_double),
        ("kmax", ctypes.c_double),
        ("n_kbin", ctypes.c_int),
        ("rmin", ctypes.c_double),
        ("rmax", ctypes.c_double),
        ("n_rbin", ctypes.c_int),
        ("periodic", ctypes.c_int),
        ("device", ctypes.c_int),
        ("fp64_stages", ctypes.c_int),
    ]


_lib = None
_lib_check = None
# the check build (device-side bounds checks, -DHG_CHECK): python hitomi_b200/build.py --check
LIB_CHECK_PATH = os.path.join(os.path.dirname(LIB_PATH), "libhitomi_b200_check.so")


def load(path: str | None = None, check: bool = False) -> ctypes.CDLL:
    """Load the library once (check=True: the check build, a separate handle).  Raises
    OSError if it has not been built."""
    global _lib, _lib_check
    if check:
        if _lib_check is None:
            _lib_check = _declare(LIB_CHECK_PATH)
        return _lib_check
    if _lib is None:
        _lib = _declare(path or LIB_PATH)
    return _lib


def _declare(p: str) -> ctypes.CDLL:
    if not os.path.exists(p):
        raise OSError(f"hitomi_b200 CUDA library not built: {p} is missing (run python hitomi_b200/build.py)")
    lib = ctypes.CDLL(p)
    c_dp = ctypes.POINTER(ctypes.c_double)
    c_ip = ctypes.POINTER(ctypes.c_int)
    vp = ctypes.c_void_p
    lib.hg_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(HgConfig)]
    lib.hg_create.restype = ctypes.c_int
    lib.hg_destroy.argtypes = [vp]
    lib.hg_destroy.restype = ctypes.c_int
    lib.hg_last_error.argtypes = [vp]
    lib.hg_last_error.restype = ctypes.c_char_p
    lib.hg_set_particles.argtypes = [vp, ctypes.c_int, c_dp, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int]
    lib.hg_set_particles.restype = ctypes.c_int
    lib.hg_set_particles_device.argtypes = lib.hg_set_particles.argtypes
    lib.hg_set_particles_device.restype = ctypes.c_int
    lib.hg_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.hg_set_profiling.restype = ctypes.c_int
    lib.hg_kernel_stats.argtypes = [vp, ctypes.c_char_p, ctypes.c_longlong]
    lib.hg_kernel_stats.restype = ctypes.c_int
    lib.hg_tuning.argtypes = [vp, ctypes.c_char_p, ctypes.c_longlong]
    lib.hg_tuning.restype = ctypes.c_int
    lib.hg_pk_box.argtypes = [vp, ctypes.c_int, c_dp, c_ip, c_dp]
    lib.hg_pk_box.restype = ctypes.c_int
    lib.hg_bk_box.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp, c_dp, c_dp]
    lib.hg_bk_box.restype = ctypes.c_int
    lib.hg_bk_box_multi.argtypes = [vp, ctypes.c_int, c_ip, ctypes.c_int, c_dp, c_dp, c_dp]
    lib.hg_bk_box_multi.restype = ctypes.c_int
    lib.hg_zeta_box.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp, c_dp, c_dp]
    lib.hg_zeta_box.restype = ctypes.c_int
    lib.hg_zeta_box_multi.argtypes = [vp, ctypes.c_int, c_ip, ctypes.c_int, c_dp, c_dp, c_dp]
    lib.hg_zeta_box_multi.restype = ctypes.c_int
    i_, d_ = ctypes.c_int, ctypes.c_double
    lib.hg_bk_survey.argtypes = [vp, i_, i_, i_, i_, d_, d_, c_dp, c_dp, c_dp]
    lib.hg_bk_survey.restype = ctypes.c_int
    lib.hg_bk_survey_multi.argtypes = [vp, i_, c_ip, i_, d_, d_, c_dp, c_dp, c_dp]
    lib.hg_bk_survey_multi.restype = ctypes.c_int
    lib.hg_zeta_survey.argtypes = lib.hg_bk_survey.argtypes
    lib.hg_zeta_survey.restype = ctypes.c_int
    lib.hg_zeta_survey_multi.argtypes = lib.hg_bk_survey_multi.argtypes
    lib.hg_zeta_survey_multi.restype = ctypes.c_int
    lib.hg_survey_scalars.argtypes = [vp, c_dp, c_dp, c_dp, c_dp, c_dp]
    lib.hg_survey_scalars.restype = ctypes.c_int
    lib.hg_pk_survey.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, c_dp, c_ip, c_dp]
    lib.hg_pk_survey.restype = ctypes.c_int
    lib.hg_xi_box.argtypes = [vp, i_, c_dp, c_ip, c_dp]
    lib.hg_xi_box.restype = ctypes.c_int
    lib.hg_xi_survey.argtypes = [vp, i_, d_, d_, c_dp, c_ip, c_dp]
    lib.hg_xi_survey.restype = ctypes.c_int
    lib.hg_xi_window.argtypes = [vp, i_, d_, c_dp, c_ip, c_dp]
    lib.hg_xi_window.restype = ctypes.c_int
    lib.hg_zeta_window.argtypes = [vp, i_, i_, i_, i_, d_, c_dp, c_dp, c_dp]
    lib.hg_zeta_window.restype = ctypes.c_int
    lib.hg_zeta_window_multi.argtypes = [vp, i_, c_ip, i_, d_, c_dp, c_dp, c_dp]
    lib.hg_zeta_window_multi.restype = ctypes.c_int
    lib.hg_reconstruct.argtypes = [vp, i_, d_, d_, d_, d_, c_dp, c_dp]
    lib.hg_reconstruct.restype = ctypes.c_int
    lib.hg_pk_box_recon.argtypes = [vp, i_, d_, c_dp, c_ip, c_dp]
    lib.hg_pk_box_recon.restype = ctypes.c_int
    lib.hg_xi_box_recon.argtypes = [vp, i_, d_, c_dp, c_ip, c_dp]
    lib.hg_xi_box_recon.restype = ctypes.c_int
    lib.hg_bk_box_recon_multi.argtypes = [vp, i_, c_ip, i_, d_, c_dp, c_dp, c_dp]
    lib.hg_bk_box_recon_multi.restype = ctypes.c_int
    lib.hg_zeta_box_recon_multi.argtypes = lib.hg_bk_box_recon_multi.argtypes
    lib.hg_zeta_box_recon_multi.restype = ctypes.c_int
    lib.hg_batch_run.argtypes = [vp, ctypes.POINTER(HgMock), i_, i_, c_ip, i_, c_ip, i_, c_ip, c_dp]
    lib.hg_batch_run.restype = ctypes.c_int
    lib.hg_batch_block_len.argtypes = [vp, i_, i_, i_]
    lib.hg_batch_block_len.restype = ctypes.c_longlong
    lib.hg_batch_done.argtypes = [vp]
    lib.hg_batch_done.restype = ctypes.c_int
    lib.hg_set_memory_limit.argtypes = [vp, ctypes.c_longlong]
    lib.hg_set_memory_limit.restype = ctypes.c_int
    lib.hg_memory_in_use.argtypes = [vp]
    lib.hg_memory_in_use.restype = ctypes.c_longlong
    lib.hg_read_ascii.argtypes = [ctypes.c_char_p, i_, ctypes.POINTER(c_dp), ctypes.POINTER(ctypes.c_longlong)]
    lib.hg_read_ascii.restype = ctypes.c_int
    lib.hg_read_gadget.argtypes = [ctypes.c_char_p, ctypes.POINTER(c_dp), ctypes.POINTER(ctypes.c_longlong),
                                   ctypes.POINTER(HgGadgetHeader)]
    lib.hg_read_gadget.restype = ctypes.c_int
    lib.hg_free.argtypes = [ctypes.c_void_p]
    lib.hg_free.restype = None
    lib.hg_pk_box_spectrum_static.argtypes = [ctypes.POINTER(HgConfig), ctypes.c_void_p, ctypes.c_longlong,
                                              ctypes.c_int, c_dp, c_ip, c_dp, ctypes.c_void_p]
    lib.hg_pk_box_spectrum_static.restype = ctypes.c_int
    lib.hg_last_timing.argtypes = [vp, c_dp, ctypes.POINTER(ctypes.c_longlong)]
    lib.hg_last_timing.restype = ctypes.c_int
    return lib
