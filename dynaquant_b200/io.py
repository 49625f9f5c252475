"""Readers for the reference's input files, so its runs can be set up unchanged.

Each reader returns numpy arrays for the Propagator setters (the file formats are the reference's;
its parsing is in systemClass.cu and sparseMatrixClasses.cu):

* read_hamiltonian  -- ``hamfile``: a MatrixMarket-style coordinate file (sparseMatrixClasses.cu:75-230):
  ``%%MatrixMarket matrix coordinate real general|symmetric|hermitian``, ``BASE_ZERO`` or ``BASE_ONE``,
  ``N N nnz``, then ``row col value`` lines.  For symmetric/hermitian files the reference hands the
  lower triangle to cuSPARSE as a symmetric matrix, so entries above the diagonal are ignored and
  those below it are mirrored.  Returns a full CSR (rowptr, col, val) with the diagonal included.
* read_ka_params -- ``ka_paramsfile``: one ``relaxTime stdDev`` line per site (systemClass.cu:982-1071);
  returns (sigma, tau) for set_noise_params.
* read_hsr_stddev -- ``hsr_stddevfile``: one standard deviation per line (systemClass.cu:912-975).
* read_initial_state -- ``initstatefile``: ``BASE_ZERO``/``BASE_ONE``, a comment line, then
  ``site amplitude`` lines up to an optional ``END``; amplitudes rounded to float as the
  reference reads them, then normalised as the reference does (systemClass.cu:1385-1481).
* read_vectors3 -- ``dipolefile`` / ``posfile``: three columns per site (spectraClass.cu:300-430).
* read_spectral_density -- ``zz_specd_file``: ``dOmega nOsc`` then ``omega J`` lines
  (systemClass.cu:1077-1207); returns (d_omega, omega, J) for set_zz_spectral_density.
"""
from __future__ import annotations

import numpy as np


def _lines(path):
    with open(path) as f:
        return [ln.rstrip("\n") for ln in f]


def read_hamiltonian(path):
    lines = _lines(path)
    head = lines[0].split()
    if len(head) < 5 or head[2] != "coordinate":
        raise ValueError(f"{path}: not a coordinate matrix file")
    kind = head[4].lower()
    if kind not in ("general", "symmetric", "hermitian"):
        raise ValueError(f"{path}: unknown matrix type {head[4]!r}")
    base = lines[1].strip()
    if base not in ("BASE_ZERO", "BASE_ONE"):
        raise ValueError(f"{path}: second line must be BASE_ZERO or BASE_ONE")
    off = 1 if base == "BASE_ONE" else 0
    n, _, nnz = (int(x) for x in lines[2].split()[:3])
    rows, cols, vals = [], [], []
    for ln in lines[3:3 + nnz]:
        p = ln.split()
        if len(p) < 3:
            continue
        i, j, v = int(p[0]) - off, int(p[1]) - off, float(p[2])
        if not (0 <= i < n and 0 <= j < n):
            raise ValueError(f"{path}: index ({i}, {j}) outside an {n} x {n} matrix")
        if kind == "general":
            rows.append(i); cols.append(j); vals.append(v)
        elif i >= j:
            rows.append(i); cols.append(j); vals.append(v)
            if i != j:
                rows.append(j); cols.append(i); vals.append(v)
    rows = np.array(rows, dtype=np.int64)
    cols = np.array(cols, dtype=np.int32)
    vals = np.array(vals, dtype=np.float64)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rowptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(rowptr, rows + 1, 1)
    return n, np.cumsum(rowptr).astype(np.int32), cols, vals


def read_ka_params(path, n):
    tau, sigma = [], []
    for ln in _lines(path):
        p = ln.split()
        if len(p) >= 2:
            tau.append(float(p[0]))
            sigma.append(float(p[1]))
    if len(tau) < n:
        raise ValueError(f"{path}: {len(tau)} sites, expected {n}")
    return np.array(sigma[:n]), np.array(tau[:n])


def read_hsr_stddev(path, n):
    vals = [float(ln.split()[0]) for ln in _lines(path) if ln.split()]
    if len(vals) < n:
        raise ValueError(f"{path}: {len(vals)} sites, expected {n}")
    return np.array(vals[:n])


def read_initial_state(path, n):
    lines = _lines(path)
    base = lines[0].strip()
    if base not in ("BASE_ZERO", "BASE_ONE"):
        raise ValueError(f"{path}: first line must be BASE_ZERO or BASE_ONE")
    off = 1 if base == "BASE_ONE" else 0
    psi = np.zeros(n, dtype=np.complex128)
    for ln in lines[2:]:
        if "END" in ln:   # the reference stops at an END line
            break
        p = ln.split()
        if len(p) >= 2:
            i = int(p[0]) - off
            if not 0 <= i < n:
                raise ValueError(f"{path}: site {i} outside 0..{n - 1}")
            # the reference reads the amplitude into a float; a later line for the same site replaces it
            psi[i] = float(np.float32(p[1]))
    nrm = np.linalg.norm(psi)
    if nrm == 0.0:
        raise ValueError(f"{path}: the state is zero")
    return psi / nrm


def read_vectors3(path):
    rows = [[float(x) for x in ln.split()[:3]] for ln in _lines(path) if len(ln.split()) >= 3]
    return np.array(rows, dtype=np.float64)


def read_spectral_density(path):
    lines = [ln.split() for ln in _lines(path) if ln.split()]
    d_omega, n_osc = float(lines[0][0]), int(lines[0][1])
    rows = np.array([[float(a), float(b)] for a, b, *_ in lines[1:1 + n_osc]])
    return d_omega, rows[:, 0], rows[:, 1]
