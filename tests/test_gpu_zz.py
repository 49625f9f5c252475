"""ZZ real noise on the GPU (dq_set_zz_spectral_density): the plain per-trajectory path and the
ensemble in FP64 and mixed precision against the FP64 oracle on the same Philox phases, and the
adjoint gradient with ZZ noise against the oracle's."""
import numpy as np
import pytest

from tests.test_noise_zz_oracle import ohmic_density

pytestmark = pytest.mark.gpu

TEMP = 300.0
POP_TOL_FP64 = 1e-10
POP_TOL_MIXED = 1e-6


def _density(oracle):
    omega, J, dw = ohmic_density()
    w, c = oracle.zz_coefficients(omega, J, dw, TEMP)
    return omega, J, dw, w, c


def _prop(s, B, steps, precision, seed=21, dt=2.0, m=12):
    import dynaquant_b200 as dq
    omega, J, dw = ohmic_density()
    p = dq.Propagator(s.n, m=m, n_traj=B, dt=dt, noise=dq.NOISE_ZZ, seed=seed, dot=dq.DOT_HERMITIAN,
                      pop_every=4, max_steps=steps, precision=precision)
    p.set_system(s)
    p.set_zz_spectral_density(omega, J, dw, TEMP)
    p.set_initial_state(s.bright_state())
    return p


def _oracle_run(oracle, s, B, steps, seed=21, dt=2.0, m=12):
    *_, w, c = _density(oracle)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=m, dt=dt, dot_mode=1, noise=oracle.NOISE_ZZ, seed=seed,
                      zz_omega=w, zz_coeff=c)
    return S.run(B, steps, s.bright_state(), pop_every=4, threads=8)


@pytest.mark.parametrize("B", [6, 5])
def test_zz_plain_and_ensemble_fp64(oracle, B):
    """24 steps cross the ensemble's 16-step noise blocks; B = 5 leaves one trajectory without a pair."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(12, 10)
    T = 24
    ref = _oracle_run(oracle, s, B, T)
    p = _prop(s, B, T, dq.PREC_FP64)
    p.run_plain(T)
    assert np.abs(p.populations() - ref["pops"]).max() <= POP_TOL_FP64
    assert np.abs(p.correlation() - ref["corr"]).max() <= POP_TOL_FP64
    p.reset()
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() <= POP_TOL_FP64
    assert np.abs(p.correlation() - ref["corr"]).max() <= POP_TOL_FP64
    p.close()


def test_zz_ensemble_mixed(oracle):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 12)
    B, T = 16, 20
    ref = _oracle_run(oracle, s, B, T)
    p = _prop(s, B, T, dq.PREC_MIXED)
    p.run(T // 2)
    p.run(T - T // 2)
    assert np.abs(p.populations() - ref["pops"]).max() <= POP_TOL_MIXED
    p.close()


def test_zz_noise_changes_with_density(oracle):
    """Re-setting the density redraws nothing but rescales: zero J gives the noiseless populations."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(12, 6)
    omega, J, dw = ohmic_density()
    p = _prop(s, 4, 8, dq.PREC_FP64)
    p.set_zz_spectral_density(omega, np.zeros_like(J), dw, TEMP)
    p.run(8)
    q = dq.Propagator(s.n, m=12, n_traj=4, dt=2.0, noise=dq.NOISE_NONE, seed=21, dot=dq.DOT_HERMITIAN,
                      pop_every=4, max_steps=8, precision=dq.PREC_FP64)
    q.set_system(s)
    q.set_initial_state(s.bright_state())
    q.run(8)
    assert np.abs(p.populations() - q.populations()).max() <= 1e-13
    with pytest.raises(dq.DQError):
        p.set_zz_spectral_density(np.zeros(3), np.ones(3), dw, TEMP)   # omega = 0: infinite amplitude
    p.close()
    q.close()


def test_zz_adjoint_matches_oracle(oracle):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    N, B, T, LEN = 48, 8, 20, 32   # 20 steps, checkpoints every 8: recomputed segments start mid-block
    s = systems.chain(N, -300.0)
    rng = np.random.default_rng(3)
    eps0 = rng.normal(0.0, 80.0, N)
    x = np.arange(N)
    psi0 = np.exp(-((x - N / 2) ** 2) / 30.0 + 0.4j * x)
    psi0 /= np.linalg.norm(psi0)
    target = rng.normal(0.0, 0.05, LEN)
    omega, J, dw, w, c = _density(oracle)
    p = dq.Propagator(N, m=12, n_traj=B, dt=2.0, noise=dq.NOISE_ZZ, seed=17, dot=dq.DOT_HERMITIAN,
                      precision=dq.PREC_FP64, max_steps=T)
    p.set_system(s)
    p.set_zz_spectral_density(omega, J, dw, TEMP)
    p.set_static_energies(eps0)
    p.set_initial_state(psi0)
    p.adjoint_setup(T, LEN, 1.0 / LEN, target, checkpoint_every=8)
    loss = p.forward()
    gs, gc = p.backward()
    rp, col, val, _ = s.off_diagonal()
    lo, go = oracle.spectrum_loss_grad(rp, col, val, s.cls_off, [1.0], eps0, 12, 2.0, psi0, B, T, LEN, 1.0 / LEN,
                                       target, seed=17, noise=oracle.NOISE_ZZ, zz_omega=w, zz_coeff=c)
    assert loss == pytest.approx(lo, rel=1e-10)
    assert np.abs(gs - go[:N]).max() <= 1e-8 * np.abs(go[:N]).max()
    assert gc[0] == pytest.approx(go[N], rel=1e-8)
    p.close()
