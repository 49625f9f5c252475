"""Parity of the batched ensemble path (shared-CSR SpMM Lanczos, batched
FP64 Padé, fused combine) with the CPU oracle: complex128 to 1e-10,
complex64 mixed precision to 1e-6 in populations."""
import numpy as np
import pytest

from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu

POP_TOL_FP64 = 1e-10
POP_TOL_MIXED = 1e-6


def _golden():
    return np.load(G.__file__.replace("make_golden.py", "golden_chain.npz"))


def _chain_prop(precision, dot, n_traj=None, steps=None):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    c = G.CHAIN
    s = systems.chain(c["n"], c["J"])
    p = dq.Propagator(s.n, m=c["m"], n_traj=n_traj or c["n_traj"], dt=c["dt"], noise=dq.NOISE_OU,
                      sigma_static=c["sigma_static"], seed=c["seed"], dot=dot, pop_every=c["pop_every"],
                      max_steps=steps or c["n_steps"], precision=precision)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, c["sigma"]), np.full(s.n, c["tau"]))
    p.set_initial_state(G.chain_psi0())
    return p


@pytest.mark.parametrize("tag,dot", [("herm", 1), ("bil", 0)])
def test_batched_fp64_matches_golden(tag, dot):
    import dynaquant_b200 as dq
    g = _golden()
    p = _chain_prop(dq.PREC_FP64, dot)
    p.run(G.CHAIN["n_steps"])
    assert np.abs(p.populations() - g[f"{tag}_pops"]).max() < POP_TOL_FP64
    assert np.abs(p.correlation() - g[f"{tag}_corr"]).max() < POP_TOL_FP64
    if tag == "herm":
        assert np.abs(p.states() - g["herm_psi_final"]).max() < 1e-10
    assert np.allclose(p.error_accum(), g[f"{tag}_err"], rtol=1e-3, atol=1e-14)
    e1, d1 = p.noise_state(1)
    assert np.array_equal(e1, g["noise_traj1_eps"]) and np.array_equal(d1, g["noise_traj1_deps"])
    p.close()


@pytest.mark.parametrize("tag,dot", [("herm", 1), ("bil", 0)])
@pytest.mark.parametrize("R", [1, 2, 4])
def test_fused_iteration_fp64_matches_golden(tag, dot, R):
    """One-kernel Lanczos iterations (staged = 2) in complex128 reproduce the golden run."""
    import dynaquant_b200 as dq
    g = _golden()
    p = _chain_prop(dq.PREC_FP64, dot)
    p.set_tiling(4, 1, 1, R, 2, 1)
    assert p.get_tiling() == (4, 1, 1, R, 2, 1)
    p.run(G.CHAIN["n_steps"])
    assert np.abs(p.populations() - g[f"{tag}_pops"]).max() < POP_TOL_FP64
    assert np.abs(p.correlation() - g[f"{tag}_corr"]).max() < POP_TOL_FP64
    assert np.allclose(p.error_accum(), g[f"{tag}_err"], rtol=1e-3, atol=1e-14)
    p.close()


def test_batched_fp64_incremental_equals_single_call():
    import dynaquant_b200 as dq
    g = _golden()
    p = _chain_prop(dq.PREC_FP64, 1)
    for k in (7, 13, 40):
        p.run(k)
    assert p.steps_done == 60
    assert np.abs(p.populations() - g["herm_pops"]).max() < POP_TOL_FP64
    p.close()


def test_batched_mixed_matches_oracle():
    import dynaquant_b200 as dq
    g = _golden()
    p = _chain_prop(dq.PREC_MIXED, 1)
    p.run(G.CHAIN["n_steps"])
    err = np.abs(p.populations() - g["herm_pops"]).max()
    assert err < POP_TOL_MIXED, err
    assert np.abs(p.correlation() - g["herm_corr"]).max() < 1e-5
    p.close()


def test_batched_mixed_tube_matches_oracle(oracle):
    """Dipole-coupled tube (480 sites, ~28 couplings/row), OU noise, 32
    trajectories x 40 steps: mixed precision vs FP64 oracle."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=20, dt=0.5, dot_mode=1, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=9)
    B, T = 32, 40
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=8, threads=4)
    for prec, tol in ((dq.PREC_MIXED, POP_TOL_MIXED), (dq.PREC_FP64, POP_TOL_FP64)):
        p = dq.Propagator(s.n, m=20, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=9, dot=1,
                          pop_every=8, max_steps=T, precision=prec)
        p.set_system(s)
        p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
        p.set_initial_state(psi0)
        p.run(T)
        err = np.abs(p.populations() - ref["pops"]).max()
        assert err < tol, (prec, err)
        assert np.abs(p.correlation() - ref["corr"]).max() < tol * 10
        p.close()


def test_batched_states_are_normalised():
    import dynaquant_b200 as dq
    p = _chain_prop(dq.PREC_MIXED, 1, n_traj=8)
    p.run(20)
    st = p.states()
    assert np.allclose(np.linalg.norm(st, axis=1), 1.0, atol=1e-12)
    p.close()


def test_spectrum_matches_numpy():
    import dynaquant_b200 as dq
    p = _chain_prop(dq.PREC_FP64, 1)
    p.run(G.CHAIN["n_steps"])
    corr = p.correlation()
    spec = p.spectrum(128)
    x = np.zeros(128, complex)
    x[:len(corr)] = corr
    assert np.abs(spec - np.fft.ifft(x) * 128).max() < 1e-10
    p.close()


@pytest.mark.parametrize("tiling", [(2, 2, 1, 1, 0, 1), (4, 1, 2, 2, 0, 1), (4, 2, 8, 4, 0, 1), (2, 1, 4, 8, 0, 2),
                                    (4, 2, 2, 8, 0, 1), (4, 2, 1, 1, 1, 1), (2, 2, 2, 1, 1, 2), (4, 1, 1, 4, 1, 1),
                                    (1, 1, 2, 4, 0, 4), (4, 2, 1, 2, 2, 1), (2, 2, 2, 1, 2, 1), (4, 1, 2, 1, 2, 1),
                                    (4, 1, 1, 3, 2, 1), (4, 2, 1, 3, 5, 1), (2, 1, 1, 2, 5, 2)])
def test_every_tiling_matches_oracle(tiling):
    """Tilings only change the schedule: each must reproduce the oracle."""
    import dynaquant_b200 as dq
    g = _golden()
    p = _chain_prop(dq.PREC_MIXED, 1)
    p.set_tiling(*tiling)
    assert p.get_tiling() == tiling
    p.run(G.CHAIN["n_steps"])
    assert np.abs(p.populations() - g["herm_pops"]).max() < POP_TOL_MIXED
    p.close()


def test_autotune_picks_valid_tiling_and_keeps_parity(tmp_path, monkeypatch):
    import dynaquant_b200 as dq
    monkeypatch.setenv("DQ_TUNE_CACHE", str(tmp_path / "tiling.json"))
    g = _golden()
    p = _chain_prop(dq.PREC_MIXED, 1)
    r = p.autotune(reps=2)
    assert not r["cached"] and r["ms_per_iter"] > 0
    assert (tmp_path / "tiling.json").exists()
    p.run(G.CHAIN["n_steps"])
    assert np.abs(p.populations() - g["herm_pops"]).max() < POP_TOL_MIXED
    p.close()
    q = _chain_prop(dq.PREC_MIXED, 1)
    r2 = q.autotune(reps=2)
    assert r2["cached"] and q.get_tiling() == (r["traj_chunk"], r["vec"], r["ctas_per_sm"], r["rows_per_block"],
                                               r["staged"], r["groups"])
    q.close()


@pytest.mark.parametrize("R,staged,groups", [(1, 1, 1), (2, 1, 1), (3, 0, 1), (4, 1, 1), (8, 1, 1), (4, 0, 1),
                                             (3, 0, 2), (2, 1, 2), (2, 0, 2), (3, 5, 1), (1, 5, 2)])
def test_tube_tilings_match_oracle(oracle, R, staged, groups):
    """Shared-memory window (TMA-staged) and L1 SpMM variants on a dipole tube,
    whose couplings reach ~3 rings (bandwidth ~60 sites)."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 40)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=12, dt=0.5, dot_mode=1, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=4)
    B, T = 32, 12
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=4, threads=4)
    p = dq.Propagator(s.n, m=12, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=4, dot=1,
                      pop_every=4, max_steps=T, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    # 16 trajectories per chunk, 2 per thread: 32 row blocks per step, so
    # R * 32 rows per staged step stays within one 256-row TMA box
    p.set_tiling(16, 2, 2, R, staged, groups)
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() < POP_TOL_MIXED
    p.close()


@pytest.mark.parametrize("tiling", [(16, 2, 2, 1, 2, 1), (16, 2, 2, 2, 2, 1), (16, 2, 1, 3, 2, 1), (16, 2, 1, 4, 2, 1),
                                    (32, 2, 1, 2, 2, 1)])
def test_tube_fused_iterations_match_oracle(oracle, tiling):
    """One-kernel Lanczos iterations (staged = 2) on the dipole tube: r_{j+1} formed from TMA-streamed
    boxes in a shared-memory ring whose halo covers the ~3-ring coupling reach."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 40)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=12, dt=0.5, dot_mode=1, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=4)
    B, T = 32, 12
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=4, threads=4)
    p = dq.Propagator(s.n, m=12, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=4, dot=1,
                      pop_every=4, max_steps=T, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    p.set_tiling(*tiling)
    assert p.get_tiling() == tiling
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() < POP_TOL_MIXED
    assert np.abs(p.correlation() - ref["corr"]).max() < POP_TOL_MIXED * 10
    p.close()


@pytest.mark.parametrize("B,tiling", [(32, (32, 1, 4, 1, 3, 1)), (32, (32, 1, 4, 2, 3, 1)), (32, (32, 1, 3, 3, 3, 1)),
                                      (64, (64, 2, 3, 3, 3, 1)), (64, (32, 1, 2, 3, 3, 2)),
                                      (32, (32, 2, 1, 1, 6, 1)), (32, (32, 2, 1, 2, 6, 1)), (32, (32, 2, 1, 3, 6, 1)),
                                      (64, (32, 2, 1, 3, 6, 1)), (32, (32, 2, 1, 1, 7, 1)), (32, (32, 2, 1, 2, 7, 1)),
                                      (32, (32, 2, 1, 3, 7, 1)), (64, (32, 2, 1, 3, 7, 1))])
def test_tube_warp_spmm_matches_oracle(oracle, B, tiling):
    """Warp-per-block SpMMs: staged = 3 gathers through L1, staged = 6 and 7 from a TMA-fed
    shared-memory ring (2 and 4 trajectories per lane); all read each block's packed records 32 at a
    time into a per-warp buffer."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 40)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=12, dt=0.5, dot_mode=1, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=4)
    T = 12
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=4, threads=4)
    p = dq.Propagator(s.n, m=12, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=4, dot=1,
                      pop_every=4, max_steps=T, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    p.set_tiling(*tiling)
    assert p.get_tiling() == tiling
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() < POP_TOL_MIXED
    assert np.abs(p.correlation() - ref["corr"]).max() < POP_TOL_MIXED * 10
    p.close()


@pytest.mark.parametrize("B,tiling", [(32, (32, 1, 1, 1, 4, 1)), (32, (32, 1, 1, 2, 4, 1)), (32, (32, 1, 1, 3, 4, 1)),
                                      (64, (64, 2, 1, 1, 4, 1)), (64, (64, 2, 1, 2, 4, 1))])
def test_tube_fused_warp_blocks_match_oracle(oracle, B, tiling):
    """Fused iteration with warp-owned row blocks (staged = 4): records in per-warp batches, gathers
    from the shared-memory ring of freshly formed residuals."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 40)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=12, dt=0.5, dot_mode=1, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=4)
    T = 12
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=4, threads=4)
    for dot in (1, 0):
        p = dq.Propagator(s.n, m=12, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=4, dot=dot,
                          pop_every=4, max_steps=T, precision=dq.PREC_MIXED)
        p.set_system(s)
        p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
        p.set_initial_state(psi0)
        p.set_tiling(*tiling)
        assert p.get_tiling() == tiling
        p.run(T)
        if dot == 1:
            assert np.abs(p.populations() - ref["pops"]).max() < POP_TOL_MIXED
            assert np.abs(p.correlation() - ref["corr"]).max() < POP_TOL_MIXED * 10
        else:   # the bilinear dot: populations stay normalised and finite
            assert np.isfinite(p.populations()).all()
        p.close()


@pytest.mark.parametrize("tag,dot", [("herm", 1), ("bil", 0)])
@pytest.mark.parametrize("R", [1, 2, 4])
def test_pform_iteration_fp64_matches_golden(tag, dot, R):
    """One launch per Lanczos iteration without the axpy pass (staged = 8, p_j = H q_{j-1} - beta q_{j-2}
    kept instead of the residual) in complex128 reproduces the golden run."""
    import dynaquant_b200 as dq
    g = _golden()
    p = _chain_prop(dq.PREC_FP64, dot)
    p.set_tiling(4, 1, 1, R, 8, 1)
    assert p.get_tiling() == (4, 1, 1, R, 8, 1)
    p.run(G.CHAIN["n_steps"])
    assert np.abs(p.populations() - g[f"{tag}_pops"]).max() < POP_TOL_FP64
    assert np.abs(p.correlation() - g[f"{tag}_corr"]).max() < POP_TOL_FP64
    assert np.allclose(p.error_accum(), g[f"{tag}_err"], rtol=1e-3, atol=1e-14)
    if tag == "herm":
        assert np.abs(p.states() - g["herm_psi_final"]).max() < 1e-10
    p.close()


@pytest.mark.parametrize("dot", [1, 0])
@pytest.mark.parametrize("tc,vec,R", [(32, 2, 3), (64, 2, 3), (32, 1, 3), (32, 2, 1), (16, 1, 2), (64, 2, 4)])
def test_pform_iteration_mixed_tube_matches_oracle(oracle, dot, tc, vec, R):
    """The same form in complex64 on the dipole-coupled tube against the FP64 oracle."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=20, dt=0.5, dot_mode=dot, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=9)
    B, T = 64, 40
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=8, threads=4)
    p = dq.Propagator(s.n, m=20, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=9, dot=dot,
                      pop_every=8, max_steps=T, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    p.set_tiling(tc, vec, 1, R, 8, 1)
    p.run(T)
    err = np.abs(p.populations() - ref["pops"]).max()
    assert err < POP_TOL_MIXED, err
    assert np.abs(p.correlation() - ref["corr"]).max() < POP_TOL_MIXED * 10
    assert np.allclose(np.linalg.norm(p.states(), axis=1), 1.0, atol=1e-12)
    p.close()


def test_pform_refuses_what_it_cannot_do():
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    p = _chain_prop(dq.PREC_MIXED, 1, n_traj=8)
    with pytest.raises(dq.DQError):
        p.set_tiling(4, 2, 1, 3, 8, 2)    # trajectory groups
    p.close()
    q = dq.Propagator(G.CHAIN["n"], m=16, n_traj=8, reorth=1, precision=dq.PREC_MIXED)
    q.set_system(systems.chain(G.CHAIN["n"], -300.0))
    q.set_initial_state(G.chain_psi0())
    with pytest.raises(dq.DQError):
        q.set_tiling(8, 2, 1, 3, 8, 1)   # full reorthogonalisation
    q.close()


@pytest.mark.parametrize("staged", [9, 10, 11])
@pytest.mark.parametrize("dot", [1, 0])
@pytest.mark.parametrize("R", [1, 2, 3])
def test_async_copy_gather_spmm_mixed_tube_matches_oracle(oracle, dot, R, staged):
    """The SpMM whose gathers are asynchronous copies into shared memory (staged = 9), the one with
    eight register gathers in flight per warp (staged = 10) and that SpMM with the axpy in the same
    cooperative launch (staged = 11), against the FP64 oracle on the dipole-coupled tube."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=20, dt=0.5, dot_mode=dot, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=9)
    B, T = 128, 40
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=8, threads=4)
    p = dq.Propagator(s.n, m=20, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=9, dot=dot,
                      pop_every=8, max_steps=T, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    p.set_tiling(64, 2, 1, R, staged, 1)
    assert p.get_tiling() == (64, 2, 1, R, staged, 1)
    p.run(T)
    err = np.abs(p.populations() - ref["pops"]).max()
    assert err < POP_TOL_MIXED, err
    assert np.abs(p.correlation() - ref["corr"]).max() < POP_TOL_MIXED * 10
    assert np.allclose(p.error_accum(), ref["err"], rtol=1e-2, atol=1e-12)
    p.close()


@pytest.mark.parametrize("staged,tc", [(11, 64), (12, 32)])
@pytest.mark.parametrize("groups", [1, 2])
def test_cooperative_iteration_chunk_groups_match_oracle(oracle, groups, staged, tc):
    """Staged 11 (SpMM and axpy in one cooperative launch, a bounded wait per chunk for alpha) and the
    lean SpMM of staged 12, with the chunks run as one launch or as two groups, against the FP64
    oracle."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=16, dt=0.5, dot_mode=1, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=21)
    B, T = 128, 24
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=4, threads=4)
    p = dq.Propagator(s.n, m=16, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=21, dot=1,
                      pop_every=4, max_steps=T, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    p.set_tiling(tc, 2, 1, 3, staged, groups)
    assert p.get_tiling() == (tc, 2, 1, 3, staged, groups)
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() < POP_TOL_MIXED
    assert np.abs(p.correlation() - ref["corr"]).max() < POP_TOL_MIXED * 10
    assert np.allclose(p.error_accum(), ref["err"], rtol=1e-2, atol=1e-12)
    p.close()


@pytest.mark.parametrize("R", [1, 2, 3])
def test_device_block_format_matches_host_builder(R):
    """The packed coupling blocks of the complex64 path are built on the device when every CSR row's
    columns are sorted, and on the host otherwise.  The same tube with each row's entries reversed
    (so the host builds the blocks) gives bit-identical populations and correlation: the two
    builders produce the same records."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    rp, col, val = np.asarray(s.rowptr), np.asarray(s.col), np.asarray(s.val)
    col_r, val_r = col.copy(), val.copy()
    for i in range(s.n):
        a, b = rp[i], rp[i + 1]
        col_r[a:b] = col[a:b][::-1]
        val_r[a:b] = val[a:b][::-1]
    B, T = 64, 12
    out = []
    for c, v in ((col, val), (col_r, val_r)):
        p = dq.Propagator(s.n, m=16, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=3, dot=1,
                          pop_every=4, max_steps=T, precision=dq.PREC_MIXED)
        p.set_hamiltonian_csr(rp, c, v)
        p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
        p.set_initial_state(s.bright_state())
        p.set_tiling(64, 2, 1, R, 5, 1)
        p.run(T)
        out.append((p.populations(), p.correlation()))
        p.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_gather_floor_probe_runs_below_the_spmm_and_refuses_other_forms():
    """dq_time_gather_floor times the gathers alone of the packed coupling blocks: it must take less time
    than the SpMM that does those gathers and more, leave the ensemble restartable, and refuse the FP64
    form (no packed records)."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(60, 100)
    B = 128
    p = dq.Propagator(s.n, m=12, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=2, dot=1,
                      pop_every=4, max_steps=8, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(s.bright_state())
    p.set_tiling(64, 2, 1, 3, 5, 1)
    floor = p.time_gather_floor(10)
    spmm = p.profile_step(1)["spmm_alpha"][0]
    assert 0.0 < floor < spmm, (floor, spmm)
    p.reset()
    p.run(4)
    assert np.allclose(p.populations()[-1].sum(), 1.0, atol=1e-6)
    p.close()
    q = dq.Propagator(s.n, m=12, n_traj=8, dt=0.5, precision=dq.PREC_FP64)
    q.set_system(s)
    q.set_initial_state(s.bright_state())
    with pytest.raises(dq.DQError):
        q.time_gather_floor(2)
    q.close()


@pytest.mark.parametrize("tc,cps", [(64, 1), (64, 2), (32, 2)])
@pytest.mark.parametrize("dot", [1, 0])
@pytest.mark.parametrize("R", [1, 2, 3])
def test_lean_spmm_mixed_tube_matches_oracle(oracle, dot, R, tc, cps):
    """The 64-register L1 SpMM (staged = 12: one 1024-thread CTA or two 512-thread CTAs per SM, 32 warps
    per SM) against the FP64 oracle on the dipole-coupled tube."""
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(20, 24)
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=20, dt=0.5, dot_mode=dot, noise=2, sigma=250.0, tau=50.0,
                      sigma_static=150.0, seed=9)
    B, T = 128, 40
    psi0 = s.bright_state()
    ref = S.run(B, T, psi0, pop_every=8, threads=4)
    p = dq.Propagator(s.n, m=20, n_traj=B, dt=0.5, noise=dq.NOISE_OU, sigma_static=150.0, seed=9, dot=dot,
                      pop_every=8, max_steps=T, precision=dq.PREC_MIXED)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(psi0)
    p.set_tiling(tc, 2, cps, R, 12, 1)
    assert p.get_tiling() == (tc, 2, cps, R, 12, 1)
    p.run(T)
    assert np.abs(p.populations() - ref["pops"]).max() < POP_TOL_MIXED
    assert np.abs(p.correlation() - ref["corr"]).max() < POP_TOL_MIXED * 10
    assert np.allclose(p.error_accum(), ref["err"], rtol=1e-2, atol=1e-12)
    p.close()
