"""Taylor-Krylov propagation (dq_set_taylor_krylov) and the inverse participation ratio
(dq_set_ipr) on the GPU against the FP64 oracle on the same noise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10


def _aux_matrix(s, rng, jitter=20.0):
    """B: the Hamiltonian's couplings with symmetric jitter and a shifted diagonal, full CSR."""
    n = s.n
    rp, col, val, diag = s.off_diagonal()
    val = val.copy()
    for i in range(n):
        for p in range(rp[i], rp[i + 1]):
            j = col[p]
            if j > i:
                d = jitter * rng.normal()
                val[p] += d
                q = [k for k in range(rp[j], rp[j + 1]) if col[k] == i][0]
                val[q] += d
    bdiag = diag + rng.normal(0.0, 15.0, n)
    frp, fcol, fval = [0], [], []
    for i in range(n):
        fcol.append(i)
        fval.append(bdiag[i])
        for p in range(rp[i], rp[i + 1]):
            fcol.append(col[p])
            fval.append(val[p])
        frp.append(len(fcol))
    return (rp, col, val, bdiag), (np.array(frp, np.int32), np.array(fcol, np.int32), np.array(fval))


def _setup(p_tk=4, m_b=10, noise=True, B=3, T=12, ipr=True):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(10, 6)
    rng = np.random.default_rng(8)
    (brp, bcol, bval, bdiag), full = _aux_matrix(s, rng)
    prop = dq.Propagator(s.n, m=12, n_traj=B, dt=2.0, noise=dq.NOISE_OU if noise else dq.NOISE_NONE, seed=13,
                         dot=dq.DOT_HERMITIAN, pop_every=3, max_steps=T, precision=dq.PREC_FP64)
    prop.set_system(s)
    if noise:
        prop.set_noise_params(np.full(s.n, 120.0), np.full(s.n, 60.0))
    prop.set_initial_state(s.bright_state())
    prop.set_taylor_krylov(p_tk, m_b, *full)
    if ipr:
        prop.set_ipr(True)
    return prop, s, (p_tk, m_b, brp, bcol, bval, bdiag)


def _oracle(oracle, s, tk, noise=True, B=3, T=12):
    rp, col, val, diag = s.off_diagonal()
    kw = dict(noise=oracle.NOISE_OU, sigma=120.0, tau=60.0) if noise else {}
    S = oracle.System(rp, col, val, diag, m=12, dt=2.0, dot_mode=1, seed=13, tk=tk, **kw)
    return S, S.run(B, T, s.bright_state(), pop_every=3, threads=4)


@pytest.mark.parametrize("p_tk,m_b", [(4, 10), (2, 16), (10, 24)])
def test_taylor_krylov_run_plain_matches_oracle(oracle, p_tk, m_b):
    prop, s, tk = _setup(p_tk, m_b)
    S, ref = _oracle(oracle, s, tk)
    prop.run_plain(12)
    assert np.abs(prop.populations() - ref["pops"]).max() <= TOL_FP64
    assert np.abs(prop.correlation() - ref["corr"]).max() <= TOL_FP64
    assert np.allclose(prop.ipr(), ref["ipr"], rtol=1e-11)
    err = prop.error_accum()
    assert np.allclose(err, ref["err"], rtol=1e-6, atol=1e-14)
    prop.close()


def test_taylor_krylov_prop_step_and_modes(oracle):
    import dynaquant_b200 as dq
    import torch
    prop, s, tk = _setup(noise=False, ipr=False)
    S, _ = _oracle(oracle, s, tk, noise=False)
    psi = torch.tensor(s.bright_state(), dtype=torch.complex128, device="cuda")
    out = torch.empty_like(psi)
    err = prop.prop_step(0, 0, psi.data_ptr(), out.data_ptr(), want_error=True)
    ref, ref_err, _ = S.tk_step(S.h0diag, s.bright_state())
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-12
    assert err == pytest.approx(ref_err, rel=1e-6)
    # the ensemble path: every (noise-free) trajectory equals two oracle steps
    prop.run(2)
    st = prop.states()
    ref2, _, _ = S.tk_step(S.h0diag, ref)
    assert np.abs(st - ref2[None, :]).max() <= 1e-12
    with pytest.raises(dq.DQError):
        prop.set_taylor_krylov(1, 8, np.zeros(s.n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    prop.set_taylor_krylov(0)          # back to Lanczos mode
    prop.run(2)
    prop.close()


@pytest.mark.parametrize("noise", [True, False])
def test_taylor_krylov_ensemble_matches_oracle(oracle, noise):
    prop, s, tk = _setup(6, 12, noise=noise, B=4)
    S, ref = _oracle(oracle, s, tk, noise=noise, B=4)
    prop.run(5)
    prop.run(7)
    assert np.abs(prop.populations() - ref["pops"]).max() <= TOL_FP64
    assert np.abs(prop.correlation() - ref["corr"]).max() <= TOL_FP64
    assert np.allclose(prop.ipr(), ref["ipr"], rtol=1e-11)
    assert np.allclose(prop.error_accum(), ref["err"], rtol=1e-6, atol=1e-14)
    # the per-trajectory path gives the same ensemble
    prop.run_plain(12)
    assert np.abs(prop.populations() - ref["pops"]).max() <= TOL_FP64
    prop.close()


@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 5e-6)])
def test_ipr_ensemble_matches_oracle(oracle, precision, tol, tmp_path):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 12)
    B, T = 16, 10
    p = dq.Propagator(s.n, m=14, n_traj=B, dt=2.0, noise=dq.NOISE_OU, seed=5, dot=dq.DOT_HERMITIAN, pop_every=5,
                      max_steps=T, precision=precision)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 150.0), np.full(s.n, 40.0))
    p.set_initial_state(s.bright_state())
    p.set_ipr(True)
    p.run(4)
    p.run(T - 4)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=14, dt=2.0, dot_mode=1, noise=oracle.NOISE_OU, sigma=150.0, tau=40.0,
                      seed=5)
    ref = S.run(B, T, s.bright_state(), pop_every=5, threads=8)
    got = p.ipr()
    assert got.shape == (T + 1,)
    assert np.abs(got / ref["ipr"] - 1).max() <= tol
    p.write_ipr(tmp_path / "invParticRat.dat")
    lines = open(tmp_path / "invParticRat.dat").read().splitlines()
    assert lines[:2] == ["# Inverse Particle Ratios", "# {timestep} {IPR}}"]
    assert len(lines) == 2 + T
    for k in (0, 3, T - 1):
        assert lines[2 + k] == "%d  %g" % (k, got[k])
    p.close()


def test_taylor_krylov_with_zz_noise(oracle):
    """Both Taylor-Krylov paths under the ZZ noise model against the oracle."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    from tests.test_noise_zz_oracle import ohmic_density
    s = systems.tube(10, 6)
    rng = np.random.default_rng(8)
    (brp, bcol, bval, bdiag), full = _aux_matrix(s, rng)
    omega, J, dw = ohmic_density()
    w, c = oracle.zz_coefficients(omega, J, dw, 300.0)
    B, T = 3, 12
    prop = dq.Propagator(s.n, m=12, n_traj=B, dt=2.0, noise=dq.NOISE_ZZ, seed=13, dot=dq.DOT_HERMITIAN, pop_every=3,
                         max_steps=T, precision=dq.PREC_FP64)
    prop.set_system(s)
    prop.set_zz_spectral_density(omega, J, dw, 300.0)
    prop.set_initial_state(s.bright_state())
    prop.set_taylor_krylov(4, 10, *full)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=12, dt=2.0, dot_mode=1, seed=13, noise=oracle.NOISE_ZZ, zz_omega=w,
                      zz_coeff=c, tk=(4, 10, brp, bcol, bval, bdiag))
    ref = S.run(B, T, s.bright_state(), pop_every=3, threads=4)
    prop.run(T)
    assert np.abs(prop.populations() - ref["pops"]).max() <= TOL_FP64
    prop.run_plain(T)
    assert np.abs(prop.populations() - ref["pops"]).max() <= TOL_FP64
    prop.close()
