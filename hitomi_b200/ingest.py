"""Catalogue readers over the C ABI (hg_read_ascii, hg_read_gadget): the reference's ASCII
survey reader (ParticleBOSSClass::readParticleBOSS, particle.hpp:93-154) and Gadget
snapshot reader (ParticleGadgetClass::readParticlesFromGagdetSnapshot,
particleGadget.hpp:211-298), native and multi-threaded."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .api import HitomiError


def _take(lib, p, n, ncols):
    try:
        return np.ctypeslib.as_array(p, shape=(n * ncols,)).reshape(n, ncols).copy() if n else np.zeros((0, ncols))
    finally:
        lib.hg_free(p)


def read_ascii(path: str, ncols: int = 4) -> np.ndarray:
    """(n, ncols) float64: every line whose first ncols fields read as numbers."""
    lib = _lib.load()
    p = ctypes.POINTER(ctypes.c_double)()
    n = ctypes.c_longlong()
    if lib.hg_read_ascii(path.encode(), int(ncols), ctypes.byref(p), ctypes.byref(n)) != 0:
        raise HitomiError(lib.hg_last_error(None).decode())
    return _take(lib, p, n.value, ncols)


def read_gadget(base: str):
    """({pos, vel * sqrt(a)} records as an (n, 6) float64 array, header) of base.0 .. base.(N-1)."""
    lib = _lib.load()
    p = ctypes.POINTER(ctypes.c_double)()
    n = ctypes.c_longlong()
    h = _lib.HgGadgetHeader()
    if lib.hg_read_gadget(base.encode(), ctypes.byref(p), ctypes.byref(n), ctypes.byref(h)) != 0:
        raise HitomiError(lib.hg_last_error(None).decode())
    return _take(lib, p, n.value, 6), h
