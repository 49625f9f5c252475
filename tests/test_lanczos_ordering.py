"""The two orders of the Lanczos subtractions agree to rounding.

The reference takes alpha_j = <q_j, H q_j>, then subtracts alpha_j q_j and
beta_{j-1} q_{j-1} (lanczosClass.cu:420-475); the oracle and the plain path keep
that order. The row-blocked ensemble SpMM starts its accumulator at
-beta_{j-1} q_{j-1} and takes alpha_j = <q_j, H q_j - beta_{j-1} q_{j-1}>
(Paige's ordering). This checks, in FP64 numpy on a tube and a random sparse
system, that both give the same tridiagonal matrix and the same propagated state
up to rounding."""
import os
import sys

import numpy as np
import pytest
import scipy.linalg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dynaquant_b200 import systems  # noqa: E402


def _lanczos(H, psi, m, paige):
    n = len(psi)
    Q = np.zeros((m + 1, n), dtype=np.complex128)
    alpha = np.zeros(m, dtype=np.complex128)
    beta = np.zeros(m)
    Q[0] = psi / np.linalg.norm(psi)
    for j in range(m):
        w = H @ Q[j]
        if paige:
            if j > 0:
                w = w - beta[j - 1] * Q[j - 1]
            alpha[j] = np.vdot(Q[j], w)
            w = w - alpha[j] * Q[j]
        else:
            alpha[j] = np.vdot(Q[j], w)
            w = w - alpha[j] * Q[j]
            if j > 0:
                w = w - beta[j - 1] * Q[j - 1]
        beta[j] = np.linalg.norm(w)
        Q[j + 1] = w / beta[j]
    return alpha, beta, Q


def _step(H, psi, m, tau, paige):
    alpha, beta, Q = _lanczos(H, psi, m, paige)
    T = np.diag(alpha) + np.diag(beta[:-1], 1) + np.diag(beta[:-1], -1)
    y = scipy.linalg.expm(tau * T)[:, 0]
    return alpha, beta, np.linalg.norm(psi) * (Q[:m].T @ y)


def _tube_hamiltonian():
    s = systems.tube(8, 12, cutoff=25.0)
    rp, col, val, diag = s.off_diagonal()
    H = np.zeros((s.n, s.n))
    for r in range(s.n):
        H[r, col[rp[r]:rp[r + 1]]] = val[rp[r]:rp[r + 1]]
    H += np.diag(diag + np.random.default_rng(3).normal(0.0, 150.0, s.n))
    return H, s.bright_state()


def _random_hamiltonian(n=200, seed=5):
    rng = np.random.default_rng(seed)
    A = np.where(rng.random((n, n)) < 0.05, rng.normal(0.0, 80.0, (n, n)), 0.0)
    H = np.triu(A, 1)
    H = H + H.T + np.diag(rng.normal(0.0, 200.0, n))
    psi = rng.normal(size=n) + 1j * rng.normal(size=n)
    return H, psi / np.linalg.norm(psi)


@pytest.mark.parametrize("make", [_tube_hamiltonian, _random_hamiltonian])
def test_paige_and_reference_orders_agree(make):
    H, psi = make()
    m = 16
    tau = -1j * 0.5 / 5308.837   # -i dt / hbar for dt = 0.5 fs, hbar in cm^-1 fs
    a0, b0, x0 = _step(H, psi, m, tau, paige=False)
    a1, b1, x1 = _step(H, psi, m, tau, paige=True)
    scale = np.abs(np.linalg.eigvalsh(H)).max()
    assert np.abs(a0 - a1).max() <= 1e-12 * scale
    assert np.abs(b0 - b1).max() <= 1e-12 * scale
    assert np.abs(x0 - x1).max() <= 1e-13
    # and both propagate like the dense exponential
    exact = scipy.linalg.expm(tau * H) @ psi
    assert np.abs(x1 - exact).max() <= 1e-10
