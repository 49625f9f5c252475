"""CPU checks of the FP64 oracle: known answers from the reference's captured
log, Random123 Philox known answers, independent scipy/numpy references and
the committed golden fixtures."""
import math

import numpy as np
import pytest
import scipy.linalg as sl

from tests.golden import make_golden as G


def test_philox_known_answers(oracle):
    # Random123 kat_vectors, philox4x32_10
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_own_log_and_sincos(oracle):
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.random(4000), np.exp(-rng.random(1000) * 36.0), [2.0 ** -53, 0.5, 0.75, 1.0]])
    for x in xs:
        ref = math.log(x)
        assert abs(oracle.log(x) - ref) <= 1e-15 * max(1.0, abs(ref))
    for u in np.concatenate([rng.random(4000), np.arange(16) / 16.0]):
        s, c = oracle.sincos_2pi(u)
        assert abs(s - math.sin(2 * math.pi * u)) < 2e-15
        assert abs(c - math.cos(2 * math.pi * u)) < 2e-15


def test_normals_are_standard(oracle):
    z = np.array([oracle.normal(99, 1, t, s, i, sub) for t in range(3) for s in range(20) for i in range(200)
                  for sub in range(2)])
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1.0) < 0.03
    # Kolmogorov-Smirnov against N(0,1)
    from scipy import stats
    assert stats.kstest(z, "norm").pvalue > 1e-3


def test_pade_ck_matches_reference_log(oracle):
    # out:82-83 (padeClass.cu:161-174 prints c_k for p = 6 with 6 significant digits)
    printed = [1, 0.5, 0.113636, 0.0151515, 0.00126263, 6.31313e-05, 1.50313e-06]
    ck = oracle.pade_ck(6)
    for a, b in zip(ck, printed):
        assert float(f"{a:.6g}") == pytest.approx(b, rel=0, abs=0)


def test_hbar_and_expcoeff_match_reference_log(oracle):
    # out:76-79: hbar_inv_cm_fs = 5308.84, neg_inv_hbar_imag.y = -0.000188365 (dt = 1)
    hb = oracle.hbar_reference()
    assert float(f"{hb:.6g}") == 5308.84
    assert float(f"{-1.0 / hb:.6g}") == -0.000188365
    import dynaquant_b200
    assert dynaquant_b200.reference_hbar() == hb


@pytest.mark.parametrize("scale", [0.05, 0.4, 3.0, 40.0])
def test_pade_exp_vs_scipy(oracle, scale):
    rng = np.random.default_rng(int(scale * 100))
    A = (rng.normal(size=(18, 18)) + 1j * rng.normal(size=(18, 18))) * scale / 18
    E, s = oracle.pade_exp(A, oracle.NORM_COMPLEX)
    ref = sl.expm(A)
    assert np.abs(E - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
    assert s >= 0


def test_pade_real_only_norm_scaling(oracle):
    # purely imaginary A: the reference's |Re| row sums give s = 0 whatever the size
    A = 1j * np.diag(np.full(6, 0.9))
    _, s_ref = oracle.pade_exp(A, oracle.NORM_REAL_ONLY)
    _, s_cx = oracle.pade_exp(A, oracle.NORM_COMPLEX)
    assert s_ref == 0 and s_cx == 1


def _chain_sys(oracle, n, dot, noise=None, **kw):
    from dynaquant_b200 import systems
    s = systems.chain(n, -300.0)
    rp, col, val, diag = s.off_diagonal()
    noise = oracle.NOISE_OU if noise is None else noise
    return oracle.System(rp, col, val, diag, m=16, dt=1.0, dot_mode=dot, noise=noise, sigma=200.0, tau=100.0,
                         sigma_static=100.0, seed=3, **kw)


@pytest.mark.parametrize("dot", [0, 1])
def test_krylov_step_vs_dense_expm(oracle, dot):
    n = 128
    S = _chain_sys(oracle, n, dot)
    eps, deps = S.traj_init(2)
    psi = np.zeros(n, complex)
    psi[n // 2] = 1
    ex = psi.copy()
    for k in range(60):
        d = S.noise_update(2, k, eps, deps)
        psi, err, nrm, s = S.krylov_step(d, psi)
        ex = sl.expm(-1j * S.dt / S.hbar * S.dense(d)) @ ex
        assert err < 1e-12
    assert np.abs(np.abs(psi) ** 2 - np.abs(ex) ** 2).max() < 1e-13
    assert abs(np.vdot(ex, psi)) == pytest.approx(1.0, abs=1e-12)


def test_lanczos_relation(oracle):
    # H Q_m = Q_m T_m + beta_m q_{m+1} e_m^T (Hermitian dot: orthonormal basis)
    n = 200
    S = _chain_sys(oracle, n, 1)
    rng = np.random.default_rng(1)
    d = rng.normal(0, 100, n)
    q1 = rng.normal(size=n) + 1j * rng.normal(size=n)
    q1 /= np.linalg.norm(q1)
    Q, al, be, nav = S.lanczos(d, q1)
    H = S.dense(d)
    m = S.m
    Qm = Q[1:m + 1].T
    T = np.diag(al[1:m + 1]) + np.diag(be[1:m].real, 1) + np.diag(be[1:m].real, -1)
    R = H @ Qm - Qm @ T
    R[:, m - 1] -= be[m].real * Q[m + 1]
    assert np.abs(R).max() < 1e-9
    assert np.abs(Qm.conj().T @ Qm - np.eye(m)).max() < 1e-10
    assert nav == pytest.approx(np.linalg.norm(H @ Q[m + 1]), rel=1e-12)


def test_full_reorthogonalisation_keeps_the_basis_orthonormal(oracle):
    """reorth = 1 (Hermitian dot): classical Gram-Schmidt against q_1..q_j after every step of the
    recurrence keeps Q orthonormal to rounding where plain Lanczos drifts, and the step still equals
    the dense exponential."""
    import scipy.linalg as sl2
    n = 200
    rng = np.random.default_rng(4)
    d = rng.normal(0, 400, n)
    q1 = rng.normal(size=n) + 1j * rng.normal(size=n)
    q1 /= np.linalg.norm(q1)
    orth = {}
    for reorth in (0, 1):
        S = _chain_sys(oracle, n, 1, reorth=reorth)
        S.m = 32
        S.s.m = 32
        Q, al, be, nav = S.lanczos(d, q1)
        Qm = Q[1:33].T
        orth[reorth] = np.abs(Qm.conj().T @ Qm - np.eye(32)).max()
        out, err, nrm, s = S.krylov_step(d, q1)
        ex = sl2.expm(-1j * S.dt / S.hbar * S.dense(d)) @ q1
        assert np.abs(out - ex).max() < 1e-10
    assert orth[1] < 1e-13
    assert orth[1] <= orth[0]


def test_ifft_matches_numpy(oracle):
    rng = np.random.default_rng(2)
    for n in (8, 64, 1024, 7, 30):
        x = rng.normal(size=n) + 1j * rng.normal(size=n)
        assert np.abs(oracle.ifft(x) - np.fft.ifft(x) * n).max() < 1e-10 * n


def test_gaussian_noise_diag(oracle):
    S = _chain_sys(oracle, 64, 1, noise=oracle.NOISE_GAUSS)
    eps, deps = S.traj_init(0)
    d = S.noise_update(0, 5, eps, deps)
    expect = np.array([oracle.normal(3, oracle.P_GAUSS, 0, 5, i, 0) * 200.0 + eps[i] for i in range(64)])
    assert np.array_equal(d, expect)


def test_golden_fixture_reproduces(oracle):
    """The oracle still produces the committed golden vectors."""
    g = np.load(G.__file__.replace("make_golden.py", "golden_chain.npz"))
    for dot, tag in ((oracle.DOT_HERMITIAN, "herm"), (oracle.DOT_BILINEAR, "bil")):
        S = G.chain_system(dot)
        r = S.run(G.CHAIN["n_traj"], G.CHAIN["n_steps"], G.chain_psi0(), pop_every=G.CHAIN["pop_every"],
                  threads=2, want_final=True)
        assert np.abs(r["pops"] - g[f"{tag}_pops"]).max() < 1e-13
        assert np.abs(r["corr"] - g[f"{tag}_corr"]).max() < 1e-13
        if tag == "herm":
            assert np.abs(r["psi_final"] - g["herm_psi_final"]).max() < 1e-12
    S = G.chain_system(oracle.DOT_HERMITIAN)
    eps, deps = S.traj_init(1)
    for k in range(G.CHAIN["n_steps"]):
        S.noise_update(1, k, eps, deps)
    assert np.array_equal(eps, g["noise_traj1_eps"]) and np.array_equal(deps, g["noise_traj1_deps"])
    vals = [oracle.normal(int(k[0]), int(k[1]), int(k[2]), int(k[3]), int(k[4]), int(k[5])) for k in g["normal_keys"]]
    assert np.array_equal(np.array(vals), g["normal_vals"])
    E, _ = oracle.pade_exp(g["pade_A"], oracle.NORM_COMPLEX)
    assert np.abs(E - g["pade_E"]).max() < 1e-15
    assert np.abs(E - sl.expm(g["pade_A"])).max() < 1e-14


def test_ensemble_populations_conserve_norm(oracle):
    S = _chain_sys(oracle, 256, 1)
    psi0 = np.zeros(256, complex)
    psi0[100] = 1
    r = S.run(3, 30, psi0, pop_every=5, threads=2)
    assert np.allclose(r["pops"].sum(1), 1.0, atol=1e-12)
    assert r["corr"][0] == pytest.approx(1.0)
    assert np.all(np.abs(r["corr"]) <= 1.0 + 1e-12)
