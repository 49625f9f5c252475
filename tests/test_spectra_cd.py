"""Absorption and circular-dichroism set-up (spectraClass.cu:300-496): initial states, the CD
correlation bra and the float scaling constants; the oracle's correlation with a separate bra
(M(0) recorded as 1, as spectraClass.cu:296 stores it)."""
import numpy as np
import pytest

from dynaquant_b200 import spectra


def _geometry(n=30, seed=4):
    rng = np.random.default_rng(seed)
    mu = rng.normal(size=(n, 3))
    R = rng.normal(scale=10.0, size=(n, 3))
    return mu, R


def test_directions_match_numpy():
    mu, R = _geometry()
    rd = np.cross(R, mu)
    ab = spectra.absorption_directions(mu)
    cd = spectra.cd_directions(mu, R)
    for d in range(3):
        m = mu[:, d] / np.linalg.norm(mu[:, d])
        k = rd[:, d] / np.linalg.norm(rd[:, d])
        assert np.allclose(ab[d][0], m, rtol=1e-15)
        assert ab[d][1] == pytest.approx(np.linalg.norm(mu[:, d]) ** 2, rel=1e-7)
        assert np.allclose(cd[d][0], k, rtol=1e-13)
        assert np.allclose(cd[d][1], m, rtol=1e-15)
        ref = np.float32(np.pi / 2 * 1e-7 * np.linalg.norm(mu[:, d]) * np.linalg.norm(rd[:, d]))
        assert cd[d][2] == pytest.approx(float(ref), rel=1e-6)


def test_oracle_correlation_with_bra(oracle):
    from dynaquant_b200 import systems
    mu, R = _geometry(n=24)
    s = systems.chain(24, -150.0)
    rp, col, val, d = s.off_diagonal()
    ket, bra, _ = spectra.cd_directions(mu, R)[1]
    S = oracle.System(rp, col, val, d, m=10, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=100.0, tau=50.0,
                      seed=6, corr_bra=bra)
    r = S.run(3, 8, ket, want_final=True)
    assert r["corr"][0] == pytest.approx(1.0)
    assert r["corr"][-1] == pytest.approx(np.mean(r["psi_final"] @ np.conj(bra)), rel=1e-12)
    # without the bra the correlation is with psi0
    S0 = oracle.System(rp, col, val, d, m=10, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=100.0, tau=50.0,
                       seed=6)
    r0 = S0.run(3, 8, ket, want_final=True)
    assert np.abs(r0["pops"] - r["pops"]).max() == 0.0
    assert r0["corr"][-1] == pytest.approx(np.mean(r0["psi_final"] @ np.conj(ket)), rel=1e-12)
