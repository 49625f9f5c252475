"""ZZ real noise in the oracle (SIM_TYPE_ZZ_REAL_NOISE; prepForZZReal, systemClass.cu:1077-1207,
and the per-step update, gpuSysHelper.cu:134-177): amplitudes, the per-step diagonal against
numpy, the phase statistics and the stationary variance of the noise."""
import numpy as np
import pytest

KB = 0.695035          # cm^-1 / K
CM_FS = 5308.84        # cm^-1 -> rad/fs


def ohmic_density(n_osc=48, d_omega=8.0, wc=120.0, lam=60.0):
    """A synthetic Ohmic spectral density J(w) = lam (w / wc) exp(-w / wc) on a grid of spacing d_omega."""
    omega = d_omega * np.arange(1, n_osc + 1)
    return omega, lam * (omega / wc) * np.exp(-omega / wc), d_omega


def test_zz_coefficients_formula(oracle):
    omega, J, dw = ohmic_density()
    T = 77.0
    w, c = oracle.zz_coefficients(omega, J, dw, T)
    G = J / (1.0 - np.exp(-omega / (KB * T)))
    assert np.allclose(w, omega / CM_FS, rtol=1e-15)
    assert np.allclose(c, np.sqrt(2.0) * np.sqrt(G * dw / np.pi), rtol=1e-14)


def _system(oracle, n=24, seed=9, T=300.0):
    from dynaquant_b200 import systems
    omega, J, dw = ohmic_density()
    w, c = oracle.zz_coefficients(omega, J, dw, T)
    s = systems.chain(n, -200.0)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=10, dt=2.0, dot_mode=1, noise=oracle.NOISE_ZZ, seed=seed,
                      zz_omega=w, zz_coeff=c)
    return S, w, c


def test_zz_diagonal_matches_numpy(oracle):
    S, w, c = _system(oracle)
    eps, _ = S.traj_init(3)
    u = S.zz_phases(3)
    assert u.dtype == np.float32 and u.min() >= 0.0 and u.max() < 1.0
    for step in (0, 1, 17, 400):
        t = step * S.dt
        ref = eps + (c[:, None] * np.cos(w[:, None] * t + 2 * np.pi * u.astype(np.float64))).sum(axis=0)
        got = S.noise_update_zz(step, eps, u)
        assert np.abs(got - ref).max() <= 1e-11 * np.abs(c).sum()
    # phases differ between trajectories and sites
    assert not np.array_equal(S.zz_phases(4), u)
    assert len(np.unique(u)) > 0.99 * u.size


def test_zz_phase_statistics_and_variance(oracle):
    S, w, c = _system(oracle, n=256)
    u = np.concatenate([S.zz_phases(t).ravel() for t in range(4)]).astype(np.float64)
    assert abs(u.mean() - 0.5) < 0.01 and abs(u.var() - 1.0 / 12) < 0.003
    # stationary variance of sum_o c_o cos(w_o t + phi_o) over random phases is sum c^2 / 2
    eps, _ = S.traj_init(0)
    x = []
    for t in range(4):
        ut = S.zz_phases(t)
        x.append(S.noise_update_zz(50, eps, ut) - eps)
    x = np.concatenate(x)
    target = (c ** 2).sum() / 2
    assert abs(x.var() / target - 1.0) < 0.15


def test_zz_run_conserves_norm(oracle):
    S, w, c = _system(oracle)
    psi0 = np.zeros(S.n, complex)
    psi0[S.n // 2] = 1.0
    r = S.run(2, 20, psi0, pop_every=5, want_final=True)
    assert np.allclose(r["pops"].sum(axis=1), 1.0, atol=1e-10)
    assert np.allclose(np.linalg.norm(r["psi_final"], axis=1), 1.0, atol=1e-10)
    # the noise moves the populations away from the noiseless run
    S0 = oracle.System(S.rowptr, S.col, S.val, S.h0diag, m=10, dt=2.0, dot_mode=1)
    r0 = S0.run(2, 20, psi0, pop_every=5)
    assert np.abs(r["pops"] - r0["pops"]).max() > 1e-3



def test_zz_coefficients_pinned_to_reference_log(oracle):
    """The reference's example run prints oscillator 0 of its spectral density (out:63-65): J = 2.08274,
    T = 77 K, omega = 0.00153248 rad/fs, G = 14.7683, coeff = 8.74586 (6 significant digits), with the
    file's spacing dOmega = 8.1357 cm^-1 also its first frequency."""
    d_omega = 8.1357
    w, c = oracle.zz_coefficients(np.array([d_omega]), np.array([2.08274]), d_omega, 77.0)
    assert float(f"{w[0]:.6g}") == 0.00153248
    assert float(f"{c[0]:.6g}") == 8.74586
    G = 2.08274 / (1.0 - np.exp(-d_omega / (KB * 77.0)))
    assert float(f"{G:.6g}") == 14.7683
