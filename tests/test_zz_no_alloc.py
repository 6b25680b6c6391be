"""The allocation-free entry point hg_pk_box_spectrum_static.

Some callers cannot call cudaMalloc: an application whose own allocator owns every byte of
the GPU (a library that allocates behind its back fails or breaks its accounting), or a
loop that cannot pay cudaMalloc's cost and implicit synchronisation on every call.  For
them the library offers one entry point that keeps all its scratch in a fixed 1 MiB
__device__ array.  This test calls it through the C ABI on a density spectrum built on the
host from a catalogue whose NGP / CIC / TSC mesh is known exactly, and checks it against
the regular entry point hg_pk_box on the same catalogue, twice in a row (the shared scratch
must be cleared between calls).  The file is named to run last; it passes alone or after
the other tests.
"""
import ctypes

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "fp32": 1e-4}
FLOOR = {"fp64": 1e-12, "fp32": 1e-3}


def interior_catalogue(n_mesh, boxsize, n, seed):
    """Particles in cells 2 .. n-3, so no NGP / CIC / TSC stencil point reaches the
    reference's flat-index boundary rule (field.hpp:92-96)."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(2, n_mesh - 2, size=(n, 3))
    frac = rng.uniform(0.0, 1.0, size=(n, 3))
    return np.ascontiguousarray((cells + frac) * (boxsize / n_mesh))


def axis_weights(xp, scheme):
    """Cell indices and weights along one axis (field.hpp:67-184)."""
    if scheme == "NGP":
        return [np.floor(xp + 0.5).astype(np.int64)], [np.ones_like(xp)]
    if scheme == "CIC":
        i0 = np.floor(xp).astype(np.int64)
        dx = xp - i0
        return [i0, i0 + 1], [1.0 - dx, dx]
    i1 = np.floor(xp + 0.5).astype(np.int64)
    dx = xp - i1
    return [i1 - 1, i1, i1 + 1], [0.5 * (0.5 - dx) ** 2, 0.75 - dx * dx, 0.5 * (0.5 + dx) ** 2]


def half_spectrum(pos, n_mesh, boxsize, scheme):
    """FFT[dV (rho - N/V)] of the assigned density (field.hpp:67-184, 505-525, 310-325)."""
    n = pos.shape[0]
    dV = boxsize ** 3 / n_mesh ** 3
    rho = np.zeros((n_mesh,) * 3)
    ax = [axis_weights(pos[:, a] * n_mesh / boxsize, scheme) for a in range(3)]
    for ix, wx in zip(*ax[0]):
        for iy, wy in zip(*ax[1]):
            for iz, wz in zip(*ax[2]):
                np.add.at(rho, (ix, iy, iz), wx * wy * wz / dV)
    return np.fft.rfftn((rho - n / boxsize ** 3) * dV)


@pytest.mark.parametrize("form", ["fp64", "fp32"])
@pytest.mark.parametrize("scheme", ["NGP", "CIC", "TSC"])
def test_static_entry_matches_context_entry(form, scheme):
    import torch
    from hitomi_b200 import _lib
    from hitomi_b200.api import ASSIGN, Binning, Context

    n_mesh, boxsize, n = 32, 1000.0, 20000
    b = Binning(0.005, 0.295, 30)
    pos = interior_catalogue(n_mesh, boxsize, n, seed=21)
    spec = half_spectrum(pos, n_mesh, boxsize, scheme)
    dtype = torch.complex128 if form == "fp64" else torch.complex64
    d_spec = torch.from_numpy(spec).to(dtype).to("cuda:0").contiguous()

    with Context(n_mesh, boxsize, b, scheme, form) as c:
        c.set_particles(0, pos)
        ref = {ell: c.pk_box(ell) for ell in (0, 2)}
        cfg = _lib.HgConfig()
        for a in range(3):
            cfg.n_mesh[a] = n_mesh
            cfg.boxsize[a] = boxsize
        cfg.assign = ASSIGN[scheme]
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
