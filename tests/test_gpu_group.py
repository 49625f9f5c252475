"""Aggregates of uneven size advanced together (dq_group_*): each member's observables equal those
of the same context run on its own, and one member matches the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T = 12


def _member(s, B, seed, m_min=0, tiling=None):
    import dynaquant_b200 as dq
    p = dq.Propagator(s.n, m=16, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=seed,
                      dot=dq.DOT_HERMITIAN, pop_every=4, max_steps=2 * T, precision=dq.PREC_MIXED, m_min=m_min,
                      m_tol=1e-7)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(s.bright_state())
    if tiling:
        p.set_tiling(*tiling)
    return p


def _systems():
    from dynaquant_b200 import systems
    return [(systems.tube(20, 40), 64, 3, 0, (32, 2, 1, 3, 6, 1)),
            (systems.tube(20, 8), 16, 4, 8, None),
            (systems.tube(20, 100), 8, 5, 0, None)]


def test_group_equals_members_run_alone(oracle):
    import dynaquant_b200 as dq
    specs = _systems()
    group_members = [_member(*sp) for sp in specs]
    g = dq.Group(group_members)
    g.run(T // 2)
    g.run(T - T // 2)
    g.close()
    for sp, pm in zip(specs, group_members):
        alone = _member(*sp)
        alone.run(T)
        assert pm.steps_done == T
        assert np.array_equal(pm.populations(), alone.populations())
        assert np.array_equal(pm.correlation(), alone.correlation())
        alone.close()
    # the first aggregate against the FP64 oracle
    s, B, seed = specs[0][0], specs[0][1], specs[0][2]
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=16, dt=0.5, dot_mode=1, noise=oracle.NOISE_OU, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=seed)
    ref = S.run(B, T, s.bright_state(), pop_every=4, threads=4)
    assert np.abs(group_members[0].populations() - ref["pops"]).max() < 1e-6
    for p in group_members:
        p.close()


def test_group_rejects_duplicates():
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    p = _member(systems.tube(20, 8), 8, 1)
    with pytest.raises(dq.DQError):
        dq.Group([p, p])
    p.close()
