"""Full reorthogonalisation (cfg.reorth = 1, Hermitian dot): the plain and batched CUDA paths against
the oracle run with the same option (classical Gram-Schmidt against q_1..q_j once per iteration)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, M, B, T = 256, 24, 8, 20


def _system():
    from dynaquant_b200 import systems
    return systems.lattice2d(16, seed=5)


def _oracle_run(oracle, s, psi0, reorth):
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=M, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=150.0, tau=60.0,
                      sigma_static=120.0, seed=13, reorth=reorth)
    return S.run(B, T, psi0, pop_every=5, threads=4)


def _prop(s, psi0, precision):
    import dynaquant_b200 as dq
    p = dq.Propagator(s.n, m=M, n_traj=B, dt=2.0, noise=dq.NOISE_OU, sigma_static=120.0, seed=13,
                      dot=dq.DOT_HERMITIAN, reorth=1, precision=precision, pop_every=5, max_steps=T)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 150.0), np.full(s.n, 60.0))
    p.set_initial_state(psi0)
    return p


def test_reorth_plain_and_batched_match_oracle(oracle):
    import dynaquant_b200 as dq
    s = _system()
    psi0 = s.bright_state((1.0, 0.0, 0.0))
    ref = _oracle_run(oracle, s, psi0, 1)
    p = _prop(s, psi0, dq.PREC_FP64)
    p.run_plain(T)
    assert np.abs(p.populations() - ref["pops"]).max() < 1e-10
    p.close()
    for prec, tol in ((dq.PREC_FP64, 1e-10), (dq.PREC_MIXED, 1e-6)):
        q = _prop(s, psi0, prec)
        q.run(T)
        assert np.abs(q.populations() - ref["pops"]).max() < tol, prec
        assert np.abs(q.correlation() - ref["corr"]).max() < tol * 10
        q.close()


def test_reorth_rejects_fused_forms_and_adjoint():
    import dynaquant_b200 as dq
    s = _system()
    psi0 = s.bright_state((1.0, 0.0, 0.0))
    p = _prop(s, psi0, dq.PREC_FP64)
    with pytest.raises(dq.DQError):
        p.set_tiling(8, 1, 1, 2, 2, 1)
    with pytest.raises(dq.DQError, match="reorth"):
        p.adjoint_setup(T, 32, 1.0, np.zeros(32))
    p.close()


@pytest.mark.parametrize("tiling", [(4, 1, 2, 2, 0, 2), (8, 1, 1, 1, 5, 1), (4, 1, 2, 4, 0, 1)])
def test_reorth_blocked_dots_under_other_tilings(oracle, tiling):
    """The one-launch dots of every h_k (blocks of 8 k, tickets per block and chunk) with trajectory
    groups, 512-thread SpMM CTAs and other row blocks, FP64, against the oracle."""
    import dynaquant_b200 as dq
    s = _system()
    psi0 = s.bright_state((1.0, 0.0, 0.0))
    ref = _oracle_run(oracle, s, psi0, 1)
    q = _prop(s, psi0, dq.PREC_FP64)
    q.set_tiling(*tiling)
    q.run(T)
    assert np.abs(q.populations() - ref["pops"]).max() < 1e-10
    assert np.abs(q.correlation() - ref["corr"]).max() < 1e-9
    q.close()
