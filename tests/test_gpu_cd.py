"""CD spectra on the GPU: the R x mu initial state with the transition-dipole bra
(dq_set_correlation_bra) on the per-trajectory, ensemble (FP64 and mixed) and Taylor-Krylov paths
against the oracle, and the overall file over the three directions (dq_write_spectrum_mean)."""
import numpy as np
import pytest

from dynaquant_b200 import spectra

pytestmark = pytest.mark.gpu

T = 12


def _geometry(n, seed=4):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, 3)), rng.normal(scale=10.0, size=(n, 3))


def _prop(s, ket, bra, precision, B=8):
    import dynaquant_b200 as dq
    p = dq.Propagator(s.n, m=12, n_traj=B, dt=2.0, noise=dq.NOISE_OU, seed=6, dot=dq.DOT_HERMITIAN, pop_every=4,
                      max_steps=T, precision=precision)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 100.0), np.full(s.n, 50.0))
    p.set_initial_state(ket)
    p.set_correlation_bra(bra)
    return p


@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 1e-6)])
def test_cd_correlation_matches_oracle(oracle, precision, tol):
    from dynaquant_b200 import systems
    s = systems.tube(12, 8)
    mu, R = _geometry(s.n)
    ket, bra, _ = spectra.cd_directions(mu, R)[2]
    rp, col, val, d = s.off_diagonal()
    S = oracle.System(rp, col, val, d, m=12, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=100.0, tau=50.0,
                      seed=6, corr_bra=bra)
    ref = S.run(8, T, ket, pop_every=4, threads=8)
    p = _prop(s, ket, bra, precision)
    p.run(T)
    assert np.abs(p.correlation() - ref["corr"]).max() <= tol
    assert np.abs(p.populations() - ref["pops"]).max() <= tol
    if precision == 0:
        p.run_plain(T)
        assert np.abs(p.correlation() - ref["corr"]).max() <= tol
    p.set_correlation_bra(None)        # back to <psi0|psi(t)>
    p.reset()
    p.run(2)
    assert p.correlation()[0] == pytest.approx(np.vdot(ket, ket).real)
    p.close()


def test_cd_spectrum_mean_file(tmp_path):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(12, 8)
    mu, R = _geometry(s.n)
    dirs = spectra.cd_directions(mu, R)
    props, corrs = [], []
    for ket, bra, sc in dirs:
        p = _prop(s, ket, bra, dq.PREC_FP64)
        p.run(T)
        props.append(p)
        corrs.append(p.correlation() * np.float32(sc))
    spectra.write_spectrum_mean(props, [d[2] for d in dirs], tmp_path / "CDCorr.dat", tmp_path / "CD.dat")
    lines = open(tmp_path / "CDCorr.dat").read().splitlines()
    mean = sum(corrs) / 3
    for i in (0, 5, T):
        parts = lines[1 + i].split()
        assert float(parts[2]) == pytest.approx(mean[i].real, rel=1e-5, abs=1e-12)
        assert float(parts[3]) == pytest.approx(mean[i].imag, rel=1e-5, abs=1e-12)
    spec = sum(np.fft.ifft(c) * len(c) for c in corrs) / 3 / T
    sl = open(tmp_path / "CD.dat").read().splitlines()
    for fid in (0, 3, T):
        parts = sl[1 + fid].split()
        assert float(parts[3]) == pytest.approx(spec[fid].real, rel=1e-5, abs=1e-12)
    for p in props:
        p.close()


def test_absorption_state_from_dipoles():
    """dq_set_initial_dipole gives psi0 = mu/|mu|: the same run as the helper's state."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(12, 8)
    mu, _ = _geometry(s.n)
    psi0, sc = spectra.absorption_directions(mu)[0]
    a = _prop(s, psi0, psi0, dq.PREC_FP64)
    a.set_correlation_bra(None)
    a.run(T)
    b = _prop(s, psi0, psi0, dq.PREC_FP64)
    b.set_correlation_bra(None)
    b.set_initial_dipole(mu[:, 0])
    b.run(T)
    assert np.abs(a.populations() - b.populations()).max() <= 1e-15
    assert np.abs(a.correlation() - b.correlation()).max() <= 1e-15
    with pytest.raises(dq.DQError):
        b.set_initial_dipole(np.zeros(s.n))
    a.close()
    b.close()


def test_cd_bra_on_taylor_krylov_paths(oracle):
    """The correlation bra on both Taylor-Krylov paths (B = the static Hamiltonian) against the oracle."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(10, 6)
    mu, R = _geometry(s.n)
    ket, bra, _ = spectra.cd_directions(mu, R)[0]
    rp, col, val, d = s.off_diagonal()
    frp, fcol, fval = s.rowptr, s.col, s.val      # B: the static Hamiltonian, diagonal included
    p = _prop(s, ket, bra, dq.PREC_FP64, B=4)
    p.set_taylor_krylov(3, 12, frp, fcol, fval)
    S = oracle.System(rp, col, val, d, m=12, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=100.0, tau=50.0,
                      seed=6, corr_bra=bra, tk=(3, 12, rp, col, val, d))
    ref = S.run(4, T, ket, pop_every=4, threads=4)
    p.run(T)
    assert np.abs(p.correlation() - ref["corr"]).max() <= 1e-10
    p.run_plain(T)
    assert np.abs(p.correlation() - ref["corr"]).max() <= 1e-10
    p.close()
