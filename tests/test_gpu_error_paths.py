"""Branches of the reference step that the benchmark configurations never
reach, and the error codes of the device status word.

* Padé scaling and squaring with s >= 2 (padeClass.cu:585-706): a time step
  large enough that ||tau Tbar||_inf lies between 2 and 8, through whole
  steps of the plain and the ensemble kernels against the oracle, whose
  Padé is itself checked against scipy's expm at that norm.
* Gaussian (HSR) noise on the ensemble path (gpuSysHelper.cu:32-66).
* DQ_ERR_NAN from a non-finite initial state, DQ_ERR_SCALING from s >= 50
  (padeClass.cu:618-623), and DQ_ERR_TIMEOUT from the TMA-fed SpMM and from
  the cooperative iteration form's per-chunk wait when a test hook makes
  their bounded waits give up on purpose.  Every failure is made on the host side: the inputs are
  ordinary numbers and every wait is bounded, so no GPU fault or hang can
  follow; after each failure the same context runs again and reproduces a
  clean run exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POP_TOL_FP64 = 1e-10
POP_TOL_MIXED = 1e-6
DQ_ERR_NAN, DQ_ERR_TIMEOUT, DQ_ERR_SCALING = 4, 5, 6


def _chain(oracle, n=256, dt=1.0, noise=2, dot=1, norm=1, seed=21):
    from dynaquant_b200 import systems
    s = systems.chain(n, -300.0)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=16, dt=dt, dot_mode=dot, norm_mode=norm, noise=noise, sigma=200.0,
                      tau=100.0, sigma_static=100.0, seed=seed)
    return s, S


def _prop(s, n_traj, dt=1.0, noise=2, dot=1, norm=1, precision=0, seed=21, **kw):
    import dynaquant_b200 as dq
    p = dq.Propagator(s.n, m=16, n_traj=n_traj, dt=dt, noise=noise, sigma_static=100.0, seed=seed, dot=dot,
                      norm=norm, precision=precision, **kw)
    p.set_system(s)
    if noise != dq.NOISE_NONE:
        p.set_noise_params(np.full(s.n, 200.0), np.full(s.n, 100.0))
    return p


# dt = 20 fs: ||tau Tbar||_inf = dt/hbar * (|alpha| + 2 beta) ~ 20/5309 * 1300 ~ 4.9, so s = 4
BIG_DT = 20.0


def test_oracle_pade_squaring_matches_expm(oracle):
    import scipy.linalg as sl
    rng = np.random.default_rng(4)
    for nrm in (2.5, 5.0, 7.5):
        A = rng.normal(size=(18, 18)) + 1j * rng.normal(size=(18, 18))
        A *= nrm / np.abs(A).sum(axis=1).max()
        E, s = oracle.pade_exp(A, oracle.NORM_COMPLEX)
        assert s >= 2
        assert np.abs(E - sl.expm(A)).max() < 1e-12 * max(1.0, np.abs(E).max())


@pytest.mark.parametrize("dot,norm", [(1, 1), (0, 1), (0, 0)])
def test_plain_step_with_pade_squaring_matches_oracle(oracle, dot, norm):
    import torch
    n = 256
    s, S = _chain(oracle, n, dt=BIG_DT, dot=dot, norm=norm)
    p = _prop(s, 2, dt=BIG_DT, dot=dot, norm=norm)
    rng = np.random.default_rng(7)
    psi0 = rng.normal(size=n) + 1j * rng.normal(size=n)   # complex: the bilinear alpha is complex
    psi0 /= np.linalg.norm(psi0)
    p.set_initial_state(psi0)
    p.reset()
    traj = 1
    eps, deps = S.traj_init(traj)
    a = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
    b = torch.empty_like(a)
    psi = psi0.copy()
    s_seen = []
    for k in range(12):
        err = p.prop_step(traj, k, a.data_ptr(), b.data_ptr(), want_error=True)
        d = S.noise_update(traj, k, eps, deps)
        psi, err_o, _, s_o = S.krylov_step(d, psi)
        s_seen.append(s_o)
        got = b.cpu().numpy()
        assert np.abs(got - psi).max() < 1e-10, (k, s_o)
        assert err == pytest.approx(err_o, rel=1e-3, abs=1e-14)
        a, b = b, a
    if norm == 1:
        assert min(s_seen) >= 2, s_seen   # the squaring branch ran in every step
    p.close()


@pytest.mark.parametrize("precision,tol", [(0, POP_TOL_FP64), (1, POP_TOL_MIXED)])
def test_ensemble_with_pade_squaring_matches_oracle(oracle, precision, tol):
    s, S = _chain(oracle, 256, dt=BIG_DT)
    B, T = 16, 24
    psi0 = np.zeros(s.n, complex)
    psi0[s.n // 2] = 1.0
    ref = S.run(B, T, psi0, pop_every=4, threads=4)
    p = _prop(s, B, dt=BIG_DT, precision=precision, pop_every=4, max_steps=T)
    p.set_initial_state(psi0)
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() < tol
    assert np.abs(p.correlation() - ref["corr"]).max() < 10 * tol
    p.close()
    # the oracle's own steps took s >= 2
    d = S.noise_update(0, 0, *S.traj_init(0))
    assert S.krylov_step(d, psi0)[3] >= 2


@pytest.mark.parametrize("precision,tol", [(0, POP_TOL_FP64), (1, POP_TOL_MIXED)])
def test_ensemble_gaussian_noise_matches_oracle(oracle, precision, tol):
    import dynaquant_b200 as dq
    s, S = _chain(oracle, 512, noise=dq.NOISE_GAUSS)
    B, T = 16, 40
    psi0 = np.zeros(s.n, complex)
    psi0[100] = 1.0
    ref = S.run(B, T, psi0, pop_every=8, threads=4)
    p = _prop(s, B, noise=dq.NOISE_GAUSS, precision=precision, pop_every=8, max_steps=T)
    p.set_initial_state(psi0)
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() < tol
    assert np.abs(p.correlation() - ref["corr"]).max() < 10 * tol
    e3, _ = p.noise_state(3)
    assert np.array_equal(e3, S.traj_init(3)[0])
    p.close()


def test_nan_initial_state_reports_nan_and_context_recovers():
    import torch

    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.chain(256, -300.0)
    good = np.zeros(s.n, complex)
    good[40] = 1.0
    bad = good.copy()
    bad[7] = np.nan
    # ensemble path
    p = _prop(s, 8, precision=dq.PREC_MIXED, max_steps=8)
    p.set_initial_state(bad)
    with pytest.raises(dq.DQError) as e:
        p.run(4)
    assert e.value.code == DQ_ERR_NAN
    p.set_initial_state(good)
    p.run(4)
    p.close()
    # drop-in step on device buffers
    p = _prop(s, 1)
    p.set_initial_state(good)
    p.reset()
    a = torch.tensor(bad, dtype=torch.complex128, device="cuda")
    b = torch.empty_like(a)
    with pytest.raises(dq.DQError) as e:
        p.prop_step(0, 0, a.data_ptr(), b.data_ptr(), want_error=True)
    assert e.value.code == DQ_ERR_NAN
    a = torch.tensor(good, dtype=torch.complex128, device="cuda")
    p.prop_step(0, 0, a.data_ptr(), b.data_ptr(), want_error=True)
    assert np.isfinite(b.cpu().numpy()).all()
    p.close()


def test_huge_time_step_reports_pade_scaling_limit():
    """s >= 50 halvings (||tau Tbar||_inf > 2^49 / 2) is refused as the reference refuses it."""
    import torch

    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.chain(256, -300.0)
    psi0 = np.zeros(s.n, complex)
    psi0[40] = 1.0
    dt = 1e18
    p = _prop(s, 8, dt=dt, noise=dq.NOISE_NONE, precision=dq.PREC_FP64, max_steps=4)
    p.set_initial_state(psi0)
    with pytest.raises(dq.DQError) as e:
        p.run(1)
    assert e.value.code == DQ_ERR_SCALING
    p.close()
    p = _prop(s, 1, dt=dt, noise=dq.NOISE_NONE)
    p.set_initial_state(psi0)
    p.reset()
    a = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
    b = torch.empty_like(a)
    with pytest.raises(dq.DQError) as e:
        p.prop_step(0, 0, a.data_ptr(), b.data_ptr(), want_error=True)
    assert e.value.code == DQ_ERR_SCALING
    p.close()


def test_ring_spmm_wait_timeout_is_reported_and_context_recovers():
    """The TMA-fed ring SpMM (staged 6) made to wait, with a budget of 20,000 cycles, on a barrier that
    nothing completes: the wait gives up, each CTA lets its own copies land and leaves, dq_run returns
    DQ_ERR_TIMEOUT; with the default budget restored the same context reproduces the clean run bit for
    bit."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    B, T = 32, 6

    def make():
        p = dq.Propagator(s.n, m=12, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=5, dot=1,
                          precision=dq.PREC_MIXED, pop_every=2, max_steps=T)
        p.set_system(s)
        p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
        p.set_initial_state(s.bright_state())
        p.set_tiling(32, 2, 1, 3, 6, 1)
        return p

    p = make()
    try:
        p.reset()
        p.run(T)
        clean = p.populations()
        p.debug_set_wait_cycles(-20000)   # a wait on a barrier that no copy completes, ~10 us
        p.reset()
        with pytest.raises(dq.DQError) as e:
            p.run(T)
        assert e.value.code == DQ_ERR_TIMEOUT
    finally:
        p.debug_set_wait_cycles(0)
    p.reset()
    p.run(T)
    assert np.array_equal(p.populations(), clean)
    p.close()


def test_cooperative_iteration_wait_timeout_is_reported_and_context_recovers():
    """Staged 11 runs the SpMM and the axpy in one cooperative launch, every block waiting (bounded)
    for its chunk's alpha.  In the forced-timeout mode that wait looks for a generation that never
    comes for 20,000 cycles: each block gives up, still takes its reduction ticket, dq_run returns
    DQ_ERR_TIMEOUT, and with the default budget restored the same context reproduces the clean run
    bit for bit."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    B, T = 64, 6
    p = dq.Propagator(s.n, m=12, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=5, dot=1,
                      precision=dq.PREC_MIXED, pop_every=2, max_steps=T)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(s.bright_state())
    p.set_tiling(64, 2, 1, 3, 11, 1)
    try:
        p.reset()
        p.run(T)
        clean = p.populations()
        p.debug_set_wait_cycles(-20000)
        p.reset()
        with pytest.raises(dq.DQError) as e:
            p.run(T)
        assert e.value.code == DQ_ERR_TIMEOUT
    finally:
        p.debug_set_wait_cycles(0)
    p.reset()
    p.run(T)
    assert np.array_equal(p.populations(), clean)
    p.close()
