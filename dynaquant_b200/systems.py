"""Seeded generators for the synthetic exciton systems (the reference's own
Hamiltonian file, data-example/hamInner.dat, is not distributed).

Each generator returns a ``System``: a full CSR (diagonal included, as the
reference's COO reader requires for a fluctuating Hamiltonian,
sparseMatrixClasses.cu:173-251), per-site transition dipoles and the
coupling class of every off-diagonal entry.

Site order is ring-major for tubes (index = ring * around + position) so the
CSR is banded and a row's neighbours sit within a few rings of it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class System:
    n: int
    rowptr: np.ndarray          # int32, n+1
    col: np.ndarray             # int32
    val: np.ndarray             # float64 (cm^-1)
    dipoles: np.ndarray         # (n, 3)
    cls_off: np.ndarray         # int32 class per off-diagonal entry, CSR order
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def off_diagonal(self):
        """(rowptr, col, val, diag) with the diagonal split out."""
        n = self.n
        rows = np.repeat(np.arange(n), np.diff(self.rowptr))
        off = rows != self.col
        diag = np.zeros(n)
        np.add.at(diag, rows[~off], self.val[~off])
        rp = np.zeros(n + 1, dtype=np.int32)
        np.cumsum(np.bincount(rows[off], minlength=n), out=rp[1:])
        return rp, self.col[off].astype(np.int32), self.val[off].copy(), diag

    def dense(self) -> np.ndarray:
        H = np.zeros((self.n, self.n))
        rows = np.repeat(np.arange(self.n), np.diff(self.rowptr))
        np.add.at(H, (rows, self.col), self.val)
        return H

    def bright_state(self, direction=(0.0, 0.0, 1.0)) -> np.ndarray:
        """psi0 = mu_dir / ||mu_dir|| (spectraClass.cu:453-455)."""
        mu = self.dipoles @ np.asarray(direction, dtype=np.float64)
        return (mu / np.linalg.norm(mu)).astype(np.complex128)


def _csr_from_pairs(n, rows, cols, vals, cls, diag):
    """Assemble a CSR with the diagonal first in each row, then couplings by column."""
    rows = np.concatenate([np.arange(n), rows])
    cols = np.concatenate([np.arange(n), cols])
    vals = np.concatenate([diag, vals])
    cls = np.concatenate([np.full(n, -1), cls])
    key = rows.astype(np.int64) * (n + 1) + np.where(rows == cols, -1, cols)
    order = np.argsort(key, kind="stable")
    rows, cols, vals, cls = rows[order], cols[order], vals[order], cls[order]
    rp = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    return rp, cols.astype(np.int32), vals.astype(np.float64), cls[rows != cols].astype(np.int32)


def chain(n=1024, J=-300.0, diag=None) -> System:
    """1-D nearest-neighbour chain, open ends."""
    i = np.arange(n - 1)
    rows = np.concatenate([i, i + 1])
    cols = np.concatenate([i + 1, i])
    vals = np.full(2 * (n - 1), float(J))
    d = np.zeros(n) if diag is None else np.asarray(diag, dtype=np.float64)
    rp, col, val, cls = _csr_from_pairs(n, rows, cols, vals, np.zeros(len(rows), dtype=np.int32), d)
    dip = np.zeros((n, 3))
    dip[:, 2] = 1.0
    return System(n, rp, col, val, dip, cls, name=f"chain{n}", meta={"J": J})


def tube(around=60, along=500, a=8.0, cutoff=25.0, C=5e4, tilt_deg=30.0) -> System:
    """Cylindrical aggregate: a square lattice of spacing a wrapped into a
    tube of `around` sites; point-dipole couplings
    J_ij = C (d_i.d_j - 3 (d_i.r)(d_j.r)) / r^3 within `cutoff` (3-D chord
    distance), dipoles tilted `tilt_deg` from the axis toward the tangent."""
    n = around * along
    R = around * a / (2 * np.pi)
    th = 2 * np.pi * (np.arange(n) % around) / around
    z = a * (np.arange(n) // around)
    pos = np.stack([R * np.cos(th), R * np.sin(th), z], 1)
    t = np.deg2rad(tilt_deg)
    tang = np.stack([-np.sin(th), np.cos(th), np.zeros(n)], 1)
    dip = np.cos(t) * np.array([0.0, 0.0, 1.0]) + np.sin(t) * tang
    rings = int(np.ceil(cutoff / a))
    rows_l, cols_l, vals_l = [], [], []
    chunk = max(1, 2_000_000 // (around * (2 * rings + 1)))
    for s in range(0, n, chunk):
        i = np.arange(s, min(n, s + chunk))
        ring = i // around
        offs = np.arange(-rings * around - around, (rings + 1) * around + around)
        j = i[:, None] + offs[None, :]
        ok = (j >= 0) & (j < n) & (j != i[:, None])
        jj = np.where(ok, j, 0)
        r = pos[jj] - pos[i][:, None, :]
        dist = np.linalg.norm(r, axis=2)
        ok &= dist < cutoff
        ok &= np.abs(jj // around - ring[:, None]) <= rings
        ii = np.broadcast_to(i[:, None], jj.shape)[ok]
        jj = jj[ok]
        r = r[ok]
        dist = dist[ok]
        rh = r / dist[:, None]
        di, dj = dip[ii], dip[jj]
        J = C * (np.sum(di * dj, 1) - 3 * np.sum(di * rh, 1) * np.sum(dj * rh, 1)) / dist ** 3
        rows_l.append(ii)
        cols_l.append(jj)
        vals_l.append(J)
    rows = np.concatenate(rows_l)
    cols = np.concatenate(cols_l)
    vals = np.concatenate(vals_l)
    rp, col, val, cls = _csr_from_pairs(n, rows, cols, vals, np.zeros(len(rows), dtype=np.int32), np.zeros(n))
    return System(n, rp, col, val, dip, cls, name=f"tube{around}x{along}",
                  meta={"around": around, "along": along, "a": a, "cutoff": cutoff, "C": C, "tilt": tilt_deg})


def lattice2d(L=64, J_nn=-250.0, J_nnn=40.0, seed=0) -> System:
    """L x L square lattice, open boundaries; nearest-neighbour couplings are
    class 0, next-nearest (diagonal) class 1.  Dipoles lie in the plane at
    seeded random angles."""
    n = L * L
    x = np.arange(n) % L
    y = np.arange(n) // L
    rows_l, cols_l, vals_l, cls_l = [], [], [], []
    for dx, dy, J, c in [(1, 0, J_nn, 0), (-1, 0, J_nn, 0), (0, 1, J_nn, 0), (0, -1, J_nn, 0),
                         (1, 1, J_nnn, 1), (-1, -1, J_nnn, 1), (1, -1, J_nnn, 1), (-1, 1, J_nnn, 1)]:
        ok = (x + dx >= 0) & (x + dx < L) & (y + dy >= 0) & (y + dy < L)
        i = np.arange(n)[ok]
        rows_l.append(i)
        cols_l.append(i + dx + dy * L)
        vals_l.append(np.full(len(i), float(J)))
        cls_l.append(np.full(len(i), c, dtype=np.int32))
    rows, cols, vals, cls = map(np.concatenate, (rows_l, cols_l, vals_l, cls_l))
    rp, col, val, cls_off = _csr_from_pairs(n, rows, cols, vals, cls, np.zeros(n))
    phi = np.random.default_rng(seed).uniform(0, 2 * np.pi, n)
    dip = np.stack([np.cos(phi), np.sin(phi), np.zeros(n)], 1)
    return System(n, rp, col, val, dip, cls_off, name=f"lattice{L}x{L}", meta={"J_nn": J_nn, "J_nnn": J_nnn})
