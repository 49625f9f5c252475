"""Parity of the plain FP64 per-trajectory CUDA path (the drop-in step)
with the CPU oracle: populations to 1e-10, noise draws bit for bit."""
import numpy as np
import pytest

from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu

POP_TOL = 1e-10   # populations, FP64 path vs FP64 oracle
PSI_TOL = 1e-11   # amplitudes


def _chain(oracle, n, dot, noise):
    from dynaquant_b200 import systems
    s = systems.chain(n, -300.0)
    rp, col, val, diag = s.off_diagonal()
    sysO = oracle.System(rp, col, val, diag, m=16, dt=1.0, dot_mode=dot, noise=noise, sigma=200.0, tau=100.0,
                         sigma_static=100.0, seed=11)
    return s, sysO


def _prop(s, n_traj, dot, noise, precision=None, **kw):
    import dynaquant_b200 as dq
    p = dq.Propagator(s.n, m=kw.pop("m", 16), n_traj=n_traj, dt=kw.pop("dt", 1.0), noise=noise,
                      sigma_static=kw.pop("sigma_static", 100.0), seed=kw.pop("seed", 11), dot=dot,
                      precision=dq.PREC_FP64 if precision is None else precision, **kw)
    p.set_system(s)
    if noise != dq.NOISE_NONE:
        p.set_noise_params(np.full(s.n, 200.0), np.full(s.n, 100.0))
    return p


@pytest.mark.parametrize("dot", [0, 1])
@pytest.mark.parametrize("noise", [1, 2])
def test_prop_step_matches_oracle(oracle, dot, noise):
    import torch
    n = 256
    s, S = _chain(oracle, n, dot, noise)
    p = _prop(s, 3, dot, noise)
    psi0 = np.zeros(n, complex)
    psi0[n // 3] = 1.0
    p.set_initial_state(psi0)
    p.reset()
    traj = 2
    eps, deps = S.traj_init(traj)
    a = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
    b = torch.empty_like(a)
    psi = psi0.copy()
    for k in range(40):
        err = p.prop_step(traj, k, a.data_ptr(), b.data_ptr(), want_error=True)
        d = S.noise_update(traj, k, eps, deps)
        psi, err_o, _, _ = S.krylov_step(d, psi)
        got = b.cpu().numpy()
        assert np.abs(got - psi).max() < PSI_TOL, k
        assert np.abs(np.abs(got) ** 2 - np.abs(psi) ** 2).max() < POP_TOL
        assert err == pytest.approx(err_o, rel=1e-3, abs=1e-15)
        a, b = b, a
    if noise == 2:
        e_gpu, d_gpu = p.noise_state(traj)
        assert np.array_equal(e_gpu, eps), "static energies differ from the oracle's Philox draws"
        assert np.array_equal(d_gpu, deps), "OU offsets differ from the oracle's Philox draws"
    p.close()


@pytest.mark.parametrize("tag,dot", [("herm", 1), ("bil", 0)])
def test_run_plain_matches_golden(tag, dot):
    import dynaquant_b200 as dq
    g = np.load(G.__file__.replace("make_golden.py", "golden_chain.npz"))
    c = G.CHAIN
    from dynaquant_b200 import systems
    s = systems.chain(c["n"], c["J"])
    p = dq.Propagator(s.n, m=c["m"], n_traj=c["n_traj"], dt=c["dt"], noise=dq.NOISE_OU,
                      sigma_static=c["sigma_static"], seed=c["seed"], dot=dot, pop_every=c["pop_every"],
                      max_steps=c["n_steps"])
    p.set_system(s)
    p.set_noise_params(np.full(s.n, c["sigma"]), np.full(s.n, c["tau"]))
    p.set_initial_state(G.chain_psi0())
    p.run_plain(c["n_steps"])
    pops = p.populations()
    corr = p.correlation()
    assert pops.shape == g[f"{tag}_pops"].shape
    assert np.abs(pops - g[f"{tag}_pops"]).max() < POP_TOL
    assert np.abs(corr - g[f"{tag}_corr"]).max() < POP_TOL
    err = p.error_accum()
    assert np.allclose(err, g[f"{tag}_err"], rtol=1e-3, atol=1e-14)
    e1, d1 = p.noise_state(1)
    assert np.array_equal(e1, g["noise_traj1_eps"]) and np.array_equal(d1, g["noise_traj1_deps"])
    p.close()


def test_tube_plain_matches_oracle(oracle):
    import torch
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)   # 480 sites, ~28 couplings per row
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=20, dt=0.5, dot_mode=1, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=5)
    p = dq.Propagator(s.n, m=20, n_traj=2, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=5, dot=1)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    psi0 = s.bright_state()
    p.set_initial_state(psi0)
    p.reset()
    eps, deps = S.traj_init(1)
    # dq_prop_step is ordered on the context's stream: create, use and read
    # the buffers on that same stream
    with torch.cuda.stream(torch.cuda.ExternalStream(p.stream)):
        a = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
        b = torch.empty_like(a)
        psi = psi0.copy()
        for k in range(25):
            p.prop_step(1, k, a.data_ptr(), b.data_ptr())
            psi, _, _, _ = S.krylov_step(S.noise_update(1, k, eps, deps), psi)
            a, b = b, a
        got = a.cpu().numpy()
    assert np.abs(np.abs(got) ** 2 - np.abs(psi) ** 2).max() < POP_TOL
    p.close()


def test_prop_step_rejects_aliasing_and_bad_traj():
    import torch
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.chain(64)
    p = dq.Propagator(64, m=8, n_traj=2)
    p.set_system(s)
    p.set_initial_state(np.eye(64)[3].astype(complex))
    a = torch.zeros(64, dtype=torch.complex128, device="cuda")
    with pytest.raises(dq.DQError) as e:
        p.prop_step(0, 0, a.data_ptr(), a.data_ptr())
    assert e.value.code == 1
    with pytest.raises(dq.DQError):
        p.prop_step(5, 0, a.data_ptr(), torch.zeros_like(a).data_ptr())
    p.close()


def test_lucky_breakdown_is_exact():
    """An invariant subspace smaller than m (uncoupled sites, psi0 on one
    site) gives beta_1 = 0.  The reference divides by zero there
    (gpuSimpleOps.cu:24-28); here q_2 = 0 decouples the rest of T and the
    step returns the exact phase exp(-i H_33 dt / hbar) e_3."""
    import torch
    import dynaquant_b200 as dq
    n = 32
    rp = np.arange(n + 1, dtype=np.int32)
    col = np.arange(n, dtype=np.int32)
    val = np.linspace(-10, 10, n)
    p = dq.Propagator(n, m=4, n_traj=1)
    p.set_hamiltonian_csr(rp, col, val)
    psi0 = np.zeros(n, complex)
    psi0[3] = 1
    p.set_initial_state(psi0)
    a = torch.tensor(psi0, device="cuda")
    b = torch.empty_like(a)
    p.prop_step(0, 0, a.data_ptr(), b.data_ptr(), want_error=True)
    out = b.cpu().numpy()
    expect = np.exp(-1j * val[3] * 1.0 / dq.reference_hbar())
    assert abs(out[3] - expect) < 1e-14
    assert np.abs(np.delete(out, 3)).max() == 0.0
    p.close()
