"""The largest workload at full size: tube 120 x 1000 = 120,000 sites, 40 A dipole cutoff (~78
couplings per row), 1024 trajectories, m = 24, OU noise 250 cm^-1 / 50 fs, static disorder 150 cm^-1,
dt = 0.5 fs.  The mixed-precision ensemble against the FP64 per-trajectory path (itself checked
against the oracle at smaller sizes) on the same Philox draws, over a few steps; size-independent
checks: population sums and |M(0)|."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T, PE, B, M = 4, 2, 1024, 24


def _prop(s, precision):
    import dynaquant_b200 as dq
    p = dq.Propagator(s.n, m=M, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=41,
                      dot=dq.DOT_HERMITIAN, precision=precision, pop_every=PE, max_steps=T)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(s.bright_state())
    return p


def test_tube_120x1000_mixed_ensemble_matches_fp64():
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(120, 1000, cutoff=40.0)
    assert s.n == 120000 and 70 < (s.nnz - s.n) / s.n < 85
    mixed = _prop(s, dq.PREC_MIXED)
    mixed.run(T)
    pm = mixed.populations()
    cm = mixed.correlation()
    mixed.close()
    ref = _prop(s, dq.PREC_FP64)
    ref.run_plain(T)
    pr = ref.populations()
    cr = ref.correlation()
    ref.close()
    assert pm.shape == (T // PE + 1, s.n)
    assert np.allclose(pm.sum(axis=1), 1.0, atol=1e-6)
    assert abs(abs(cm[0]) - 1.0) < 1e-12
    assert np.abs(pm - pr).max() <= 1e-6
    assert np.abs(cm - cr).max() <= 1e-5


def test_tube_120x1000_states_match_oracle(oracle):
    """The same 120,000-site tube (m = 24, ~78 couplings per row) against the FP64 oracle itself: the
    ensemble in complex64 under the tiling the autotuner picks for it (64 trajectories per chunk, 2 per
    lane, 3 rows per block, the 512-thread L1 SpMM) and in complex128, two steps, compared state by
    state on trajectories 0 and 1 (the Philox draws are keyed by the global trajectory index, so they are
    the oracle's trajectories 0 and 1 whatever the ensemble size)."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(120, 1000, cutoff=40.0)
    rp, col, val, diag = s.off_diagonal()
    steps, nt = 2, 2
    S = oracle.System(rp, col, val, diag, m=M, dt=0.5, dot_mode=oracle.DOT_HERMITIAN, noise=oracle.NOISE_OU,
                      sigma=250.0, tau=50.0, sigma_static=150.0, seed=41)
    ref = S.run(nt, steps, s.bright_state(), pop_every=1, threads=nt, want_final=True)["psi_final"]
    for prec, tol in ((dq.PREC_MIXED, 1e-5), (dq.PREC_FP64, 1e-10)):
        p = dq.Propagator(s.n, m=M, n_traj=64, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=41,
                          dot=dq.DOT_HERMITIAN, precision=prec, pop_every=1, max_steps=steps)
        p.set_system(s)
        p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
        p.set_initial_state(s.bright_state())
        if prec == dq.PREC_MIXED:
            p.set_tiling(64, 2, 1, 3, 5, 1)
        p.run(steps)
        st = p.states()[:nt]
        p.close()
        rel = np.abs(st - ref).max() / np.abs(ref).max()
        print(f"tube 120x1000 {'mixed' if prec == dq.PREC_MIXED else 'FP64'} vs oracle, states of "
              f"{nt} trajectories after {steps} steps: max|dpsi| / max|psi| = {rel:.3e}")
        assert rel < tol, (prec, rel)
