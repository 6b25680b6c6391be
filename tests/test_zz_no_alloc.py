"""The allocation-free entry point hg_pk_box_spectrum_static.

Some callers cannot call cudaMalloc: work captured into a CUDA graph, where allocation is
not allowed, or an application whose allocator owns every byte of the GPU.  For them the
library offers one entry point that keeps all its scratch in a fixed 1 MiB __device__
array.  This test calls it through the C ABI on a density spectrum built from a catalogue
whose mesh is known exactly, and checks it against the regular entry point hg_pk_box on
the same catalogue, twice in a row (the shared scratch must be cleared between calls).
The file is named to run last; it passes alone or after the other tests.
"""
import ctypes

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}


def exact_ngp_catalogue(n_mesh, boxsize, n, seed):
    """Particles strictly inside interior cells, so NGP assignment is exact counting and
    no stencil point reaches the reference's flat-index boundary rule."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(1, n_mesh - 1, size=(n, 3))
    frac = rng.uniform(-0.3, 0.3, size=(n, 3))
    pos = (cells + frac) * (boxsize / n_mesh)
    return np.ascontiguousarray(pos), cells


def half_spectrum(cells, n_mesh, boxsize, n):
    """FFT[dV (rho - N/V)] of the NGP density (field.hpp:67-100, 505-525, 310-325)."""
    ntot = n_mesh ** 3
    dV = boxsize ** 3 / ntot
    factor = 1.0 / dV
    rho = np.zeros((n_mesh,) * 3)
    np.add.at(rho, (cells[:, 0], cells[:, 1], cells[:, 2]), factor)
    field = (rho - n / boxsize ** 3) * dV
    return np.fft.rfftn(field)


@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_static_entry_matches_context_entry(form):
    import torch
    from hitomi_b200 import _lib
    from hitomi_b200.api import Binning, Context

    n_mesh, boxsize, n = 32, 1000.0, 20000
    b = Binning(0.005, 0.295, 30)
    pos, cells = exact_ngp_catalogue(n_mesh, boxsize, n, seed=21)
    spec = half_spectrum(cells, n_mesh, boxsize, n)
    dtype = torch.complex128 if form == "fp64" else torch.complex64
    d_spec = torch.from_numpy(spec).to(dtype).to("cuda:0").contiguous()

    with Context(n_mesh, boxsize, b, "NGP", form) as c:
        c.set_particles(0, pos)
        ref = {ell: c.pk_box(ell) for ell in (0, 2)}
        cfg = _lib.HgConfig()
        for a in range(3):
            cfg.n_mesh[a] = n_mesh
            cfg.boxsize[a] = boxsize
        cfg.assign = _lib.HG_NGP
        cfg.precision = _lib.HG_FP64 if form == "fp64" else _lib.HG_FP32
        cfg.kmin, cfg.kmax, cfg.n_kbin = b.kmin, b.kmax, b.n_kbin
        cfg.rmin, cfg.rmax, cfg.n_rbin = b.rmin, b.rmax, b.n_rbin
        cfg.device = 0
        lib = _lib.load()
        for ell in (0, 2):  # two calls in a row on the shared scratch
            out = np.zeros(2 * b.n_kbin)
            nmode = np.zeros(b.n_kbin, dtype=np.int32)
            norm = ctypes.c_double()
            rc = lib.hg_pk_box_spectrum_static(ctypes.byref(cfg), ctypes.c_void_p(d_spec.data_ptr()), n, ell,
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               nmode.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                               ctypes.byref(norm), None)
            assert rc == 0, lib.hg_last_error(None).decode()
            pk_ref, nmode_ref, norm_ref = ref[ell]
            pk = out[0::2] + 1j * out[1::2]
            np.testing.assert_array_equal(nmode, nmode_ref)
            assert norm.value == norm_ref
            assert relerr(norm.value * pk, norm_ref * pk_ref, FLOOR[form]) < TOL[form], ell


def test_static_entry_rejects_oversized_requests():
    import torch
    from hitomi_b200 import _lib

    lib = _lib.load()
    cfg = _lib.HgConfig()
    for a in range(3):
        cfg.n_mesh[a] = 32
        cfg.boxsize[a] = 1000.0
    cfg.assign, cfg.precision = _lib.HG_TSC, _lib.HG_FP64
    cfg.kmin, cfg.kmax, cfg.n_kbin = 0.01, 0.3, 257  # more bins than the scratch holds
    cfg.rmin, cfg.rmax, cfg.n_rbin = 10.0, 100.0, 10
    d = torch.zeros(32 * 32 * 17, dtype=torch.complex128, device="cuda:0")
    out = np.zeros(2 * 257)
    rc = lib.hg_pk_box_spectrum_static(ctypes.byref(cfg), ctypes.c_void_p(d.data_ptr()), 1000, 0,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None, None, None)
    assert rc == -1
    assert "n_kbin" in lib.hg_last_error(None).decode()
