"""Initial states, correlation bras and scaling constants of the reference's absorption and
circular-dichroism (CD) spectra (spectraClass.cu), one polarisation direction per run.

The reference reads per-site transition dipoles mu_i (and, for CD, positions R_i) from files
(spectraClass.cu:300-430); for direction d it propagates
  absorption: psi0 = mu_d / |mu_d|, correlation <psi0|psi(t)>, scaling |mu_d|^2;
  CD:         psi0 = (R x mu)_d / |(R x mu)_d|, correlation <mu_d / |mu_d| | psi(t)>,
              scaling (pi/2) 1e-7 |mu_d| |(R x mu)_d|
(prepInitState :432-496, calcCorrFunc :505-571, the scaling constants :640-651, which the
reference holds in a float).  The per-direction files come from Propagator.write_spectrum and
the overall mean from write_spectrum_mean.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _norms(v):
    # sqrt of the sum of squares per direction (spectraClass.cu:400-411)
    return np.sqrt((v * v).sum(axis=0))


def absorption_directions(dipoles):
    """[(psi0, scaling)] for x, y, z from the (N, 3) transition dipoles."""
    mu = np.asarray(dipoles, dtype=np.float64)
    mu_tot = _norms(mu)
    out = []
    for d in range(3):
        psi0 = (mu[:, d] / mu_tot[d]).astype(np.complex128)
        out.append((psi0, float(np.float32(mu_tot[d] ** 2))))
    return out


def cd_directions(dipoles, positions):
    """[(psi0, bra, scaling)] for x, y, z: psi0 from R x mu, the bra from mu (spectraClass.cu:356-385)."""
    mu = np.asarray(dipoles, dtype=np.float64)
    R = np.asarray(positions, dtype=np.float64)
    rd = np.stack([R[:, 1] * mu[:, 2] - R[:, 2] * mu[:, 1],
                   R[:, 2] * mu[:, 0] - R[:, 0] * mu[:, 2],
                   R[:, 0] * mu[:, 1] - R[:, 1] * mu[:, 0]], axis=1)
    mu_tot, rd_tot = _norms(mu), _norms(rd)
    pi_half = np.float32(np.float32(3.1415926535) / np.float32(2.0))
    out = []
    for d in range(3):
        sc = np.float32(float(pi_half) * 10.0 ** -7)
        sc = np.float32(float(sc) * (mu_tot[d] * rd_tot[d]))
        out.append(((rd[:, d] / rd_tot[d]).astype(np.complex128), (mu[:, d] / mu_tot[d]).astype(np.complex128),
                    float(sc)))
    return out


def write_spectrum_mean(props, scalings, corr_path, spec_path):
    """The overall correlation and spectrum files: the mean over the directions' contexts."""
    L = _lib.load()
    arr = (C.c_void_p * len(props))(*[p.h for p in props])
    sc = np.ascontiguousarray(scalings, dtype=np.float64)
    rc = L.dq_write_spectrum_mean(arr, len(props), _lib.dptr(sc), str(corr_path).encode(), str(spec_path).encode())
    if rc != 0:
        raise _lib.DQError(rc, L.dq_last_error(props[0].h).decode(errors="replace"))
