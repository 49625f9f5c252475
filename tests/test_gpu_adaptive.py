"""Adaptive Krylov dimension (cfg.m_min > 0): each trajectory takes the first checked dimension
j = m_min, m_min + 4, ... whose EXPOKIT term beta_j |E(j-1, j)| meets m_tol (else m).  The batched
path against the oracle with the same rule, and the per-chunk early exit under several tilings."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M_MAX, M_MIN, TOL, B, T, DT = 24, 8, 1e-9, 32, 10, 20.0


def _setup(oracle):
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    rp, col, val, diag = s.off_diagonal()
    # dt = 20 fs: trajectories and steps choose 16 or 20
    S = oracle.System(rp, col, val, diag, m=M_MAX, dt=DT, dot_mode=1, norm_mode=1, noise=oracle.NOISE_OU,
                      sigma=250.0, tau=50.0, sigma_static=150.0, seed=21, m_min=M_MIN, m_tol=TOL)
    return s, S


def _oracle_dims(S, psi0):
    """Dimensions the oracle chooses for trajectories 0-3 over the run (to show they vary)."""
    ms = []
    for traj in range(4):
        eps, deps = S.traj_init(traj)
        psi = psi0.copy()
        for k in range(T):
            d = S.noise_update(traj, k, eps, deps)
            psi, _, mu = S.krylov_step_m(d, psi)
            ms.append(mu)
    return ms


@pytest.mark.parametrize("precision,tiling", [("fp64", None), ("mixed", None), ("mixed", (32, 2, 1, 3, 6, 1)),
                                              ("mixed", (8, 2, 2, 3, 0, 2)), ("mixed", (8, 2, 1, 3, 12, 2))])
def test_adaptive_dimension_matches_oracle(oracle, precision, tiling):
    import dynaquant_b200 as dq
    s, S = _setup(oracle)
    psi0 = s.bright_state()
    ms = _oracle_dims(S, psi0)
    assert min(ms) < M_MAX and len(set(ms)) > 1, ms
    ref = S.run(B, T, psi0, pop_every=2, threads=4)
    p = dq.Propagator(s.n, m=M_MAX, n_traj=B, dt=DT, noise=dq.NOISE_OU, sigma_static=150.0, seed=21,
                      dot=dq.DOT_HERMITIAN, norm=dq.NORM_COMPLEX, pop_every=2, max_steps=T,
                      precision=dq.PREC_FP64 if precision == "fp64" else dq.PREC_MIXED, m_min=M_MIN, m_tol=TOL)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    if tiling:
        p.set_tiling(*tiling)
    p.run(T)
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert np.abs(p.populations() - ref["pops"]).max() < tol
    assert np.abs(p.correlation() - ref["corr"]).max() < 10 * tol
    if precision == "fp64":
        # the accumulated err1 terms match only when every trajectory chose the same dimensions
        assert np.allclose(p.error_accum(), ref["err"], rtol=1e-3, atol=1e-13)
    p.close()


def test_adaptive_rejects_fused_forms():
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    p = dq.Propagator(s.n, m=M_MAX, n_traj=B, dt=DT, precision=dq.PREC_MIXED, m_min=M_MIN, m_tol=TOL)
    p.set_system(s)
    p.set_initial_state(s.bright_state())
    with pytest.raises(dq.DQError):
        p.set_tiling(16, 2, 2, 2, 2, 1)
    p.close()
