"""Taylor-Krylov propagation (taylorKrylovClass.cu:135-434) in the oracle: the Taylor sum plus the
phi_p Krylov term on an auxiliary matrix B, checked against dense matrix functions; and the inverse
participation ratio (systemClass.cu:2219-2257) of the oracle's ensemble run."""
import math

import numpy as np
import pytest
import scipy.linalg as sla


def _chain_csr(n, J, rng=None, jitter=0.0):
    rp, col, val = [0], [], []
    for i in range(n):
        for j in (i - 1, i + 1):
            if 0 <= j < n:
                col.append(j)
                val.append(J + (jitter * rng.normal() if rng is not None else 0.0))
        rp.append(len(col))
    # symmetrise jittered couplings
    val = np.array(val)
    if jitter:
        for i in range(n):
            for p in range(rp[i], rp[i + 1]):
                j = col[p]
                if j > i:
                    q = [k for k in range(rp[j], rp[j + 1]) if col[k] == i][0]
                    val[q] = val[p]
    return np.array(rp, np.int32), np.array(col, np.int32), val


def _dense(rp, col, val, diag):
    n = len(diag)
    H = np.diag(diag).astype(float)
    for i in range(n):
        for p in range(rp[i], rp[i + 1]):
            H[i, col[p]] += val[p]
    return H


def _setup(oracle, n=14, p=4, mb=14, b_jitter=15.0, dot=1):
    rng = np.random.default_rng(2)
    rp, col, val = _chain_csr(n, -120.0)
    diag = rng.normal(0, 80.0, n)
    brp, bcol, bval = _chain_csr(n, -120.0, rng, b_jitter)
    bdiag = diag + rng.normal(0, 10.0, n)
    S = oracle.System(rp, col, val, diag, m=10, dt=4.0, dot_mode=dot,
                      tk=(p, mb, brp, bcol, bval, bdiag))
    psi = rng.normal(size=n) + 1j * rng.normal(size=n)
    psi /= np.linalg.norm(psi)
    return S, diag, psi, _dense(rp, col, val, diag), _dense(brp, bcol, bval, bdiag)


@pytest.mark.parametrize("p", [2, 3, 6])
def test_tk_matches_dense_formula(oracle, p):
    S, diag, psi, A, Bm = _setup(oracle, p=p)
    tau = -1j * S.dt / S.hbar
    out, err, nrm = S.tk_step(diag, psi)
    taylor = sum((tau ** k / math.factorial(k)) * np.linalg.matrix_power(A, k) @ psi for k in range(p))
    v = np.linalg.matrix_power(A, p) @ psi
    beta0 = np.linalg.norm(v)
    # the phi term of exp(tau Tbar) in its tau-scaled form: exp of tau * [[B, e, 0], [0, 0, 1], ...]
    n = len(psi)
    M = np.zeros((n + p, n + p), complex)
    M[:n, :n] = Bm
    M[:n, n] = v / beta0
    for k in range(p - 1):
        M[n + k, n + k + 1] = 1.0
    krylov = beta0 * sla.expm(tau * M)[:n, n + p - 1]
    ref = taylor + krylov
    assert nrm == pytest.approx(np.linalg.norm(ref), rel=1e-11)
    assert np.abs(out - ref / np.linalg.norm(ref)).max() < 1e-11
    assert err >= 1.1e-16


def test_tk_with_b_equal_a_is_the_exponential(oracle):
    """exp(tau A) v = sum_{k<p} tau^k/k! A^k v + tau^p phi_p(tau A) A^p v exactly."""
    n = 14
    rng = np.random.default_rng(4)
    rp, col, val = _chain_csr(n, -150.0)
    diag = rng.normal(0, 60.0, n)
    S = oracle.System(rp, col, val, diag, m=14, dt=3.0, dot_mode=1, tk=(5, 14, rp, col, val, diag))
    psi = np.zeros(n, complex)
    psi[n // 2] = 1.0
    out, err, nrm = S.tk_step(diag, psi)
    A = _dense(rp, col, val, diag)
    ref = sla.expm(-1j * S.dt / S.hbar * A) @ psi
    assert abs(nrm - 1.0) < 1e-11
    assert np.abs(out - ref).max() < 1e-11
    # the Lanczos-mode step agrees
    L = oracle.System(rp, col, val, diag, m=14, dt=3.0, dot_mode=1)
    out_l, *_ = L.krylov_step(diag, psi)
    assert np.abs(out - out_l).max() < 1e-11


def test_tk_zero_b_is_the_taylor_polynomial(oracle):
    """B = 0: phi_p(0) = 1/p!, so the step is the order-p Taylor polynomial of exp(tau A)."""
    n, p = 10, 3
    rng = np.random.default_rng(5)
    rp, col, val = _chain_csr(n, -90.0)
    diag = rng.normal(0, 40.0, n)
    zrp = np.zeros(n + 1, np.int32)
    S = oracle.System(rp, col, val, diag, m=8, dt=2.0, dot_mode=1,
                      tk=(p, 6, zrp, np.zeros(0, np.int32), np.zeros(0), np.zeros(n)))
    psi = rng.normal(size=n) + 0j
    psi /= np.linalg.norm(psi)
    out, _, nrm = S.tk_step(diag, psi)
    A = _dense(rp, col, val, diag)
    tau = -1j * S.dt / S.hbar
    ref = sum((tau ** k / math.factorial(k)) * np.linalg.matrix_power(A, k) @ psi for k in range(p + 1))
    assert nrm == pytest.approx(np.linalg.norm(ref), rel=1e-12)
    assert np.abs(out - ref / np.linalg.norm(ref)).max() < 1e-12


def test_tk_ensemble_run_and_ipr(oracle):
    S, diag, psi, A, Bm = _setup(oracle, p=4, mb=8)
    r = S.run(3, 6, psi, pop_every=2, want_final=True)
    assert np.allclose(r["pops"].sum(axis=1), 1.0, atol=1e-12)
    # trajectories are identical without noise: step by step against tk_step
    x = psi.copy()
    iprs = [1.0 / (np.abs(x) ** 4).sum()]
    for k in range(6):
        x, _, _ = S.tk_step(S.h0diag, x)
        iprs.append(1.0 / (np.abs(x) ** 4).sum())
    assert np.allclose(r["ipr"], iprs, rtol=1e-12)
    assert np.abs(r["psi_final"][0] - x).max() < 1e-12


def test_ipr_of_lanczos_run(oracle):
    from dynaquant_b200 import systems
    s = systems.chain(32, -200.0)
    rp, col, val, d = s.off_diagonal()
    S = oracle.System(rp, col, val, d, m=10, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=100.0, tau=50.0,
                      seed=3)
    psi0 = np.zeros(32, complex)
    psi0[16] = 1.0
    r = S.run(4, 8, psi0, want_final=True)
    assert r["ipr"][0] == pytest.approx(1.0)
    fin = r["psi_final"]
    assert r["ipr"][-1] == pytest.approx(np.mean(1.0 / (np.abs(fin) ** 4).sum(axis=1)), rel=1e-12)
    assert (r["ipr"][1:] > 1.0).all()     # the excitation spreads
