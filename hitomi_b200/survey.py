"""Host-side preparation of survey catalogues, as the reference's survey driver does it
before any estimator runs (src/hitomi_measurement/main.cpp:129-180):

  * line of sight per particle, los = pos / |pos| with the observer at the origin
    (ParticleBOSSClass::calcLOS, particle.hpp:355-372);
  * both catalogues shifted so that the randoms' minimum sits `factor` cells inside the
    FFT box (ParticleBOSSClass::resetParticleForFFT, particle.hpp:222-262; the driver
    calls it with its default factor 1, main.cpp:171-175 and, after a reconstruction,
    main.cpp:220).

The result is the reference's array of structs {pos[3], los[3], w} (56 bytes per
particle, particle.hpp:12-16), which the library reads in place (pos_off 0, los_off 3,
w_off 6).  Every expression keeps the reference's operation order, so the records are
bit-identical to the ones its estimators see.
"""
from __future__ import annotations

import numpy as np

POS_OFF, LOS_OFF, W_OFF = 0, 3, 6


def records(xyzw: np.ndarray) -> np.ndarray:
    """(n, 4) x y z w -> (n, 7) {pos, los, w} with los = pos / |pos|."""
    a = np.asarray(xyzw, dtype=np.float64)
    x, y, z = a[:, 0], a[:, 1], a[:, 2]
    mag = np.sqrt(x * x + y * y + z * z)
    out = np.empty((a.shape[0], 7))
    out[:, 0:3] = a[:, 0:3]
    out[:, 3] = x / mag
    out[:, 4] = y / mag
    out[:, 5] = z / mag
    out[:, 6] = a[:, 3]
    return out


def shift_into_box(D: np.ndarray, R: np.ndarray, n_mesh, boxsize, factor: float = 1.0):
    """Subtract dP = min(R.pos) - factor * boxsize / n_mesh from both catalogues' positions
    (in place); returns dP."""
    nm = np.broadcast_to(np.asarray(n_mesh, dtype=np.float64), (3,))
    bs = np.broadcast_to(np.asarray(boxsize, dtype=np.float64), (3,))
    dP = R[:, 0:3].min(axis=0).copy()
    for a in range(3):
        dP[a] -= factor * bs[a] / nm[a]
    D[:, 0:3] -= dP
    R[:, 0:3] -= dP
    return dP


def prepare(data_xyzw: np.ndarray, rand_xyzw: np.ndarray, n_mesh, boxsize, factor: float = 1.0):
    """The reference driver's preparation of (data, randoms): records with LOS, then the shift."""
    D, R = records(data_xyzw), records(rand_xyzw)
    shift_into_box(D, R, n_mesh, boxsize, factor)
    return np.ascontiguousarray(D), np.ascontiguousarray(R)
