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
