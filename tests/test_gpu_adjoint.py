"""Adjoint gradient of the spectrum-fitting loss on the GPU (dq_adjoint_setup / dq_forward /
dq_backward) against the FP64 oracle's adjoint (itself checked against finite differences on the
CPU), against finite differences of the GPU's own forward loss, and checkpointed recomputation
against keeping every step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, M, B, T, LEN = 64, 12, 8, 12, 16
DT, SIGMA, TAU, SEED = 2.0, 60.0, 80.0, 31
GRAD_TOL_FP64 = 1e-8     # relative to max |gradient|
GRAD_TOL_MIXED = 3e-4
FD_TOL = 1e-5


def _problem():
    from dynaquant_b200 import systems
    s = systems.chain(N, -300.0)
    rng = np.random.default_rng(5)
    eps0 = rng.normal(0.0, 100.0, N)
    x = np.arange(N)
    psi0 = np.exp(-((x - N / 2) ** 2) / 30.0 + 0.4j * x)
    psi0 /= np.linalg.norm(psi0)
    target = rng.normal(0.0, 0.05, LEN)
    return s, eps0, psi0, target


def _prop(precision, s, eps0, psi0, target, scale_c=None, ck=0, noise=True):
    import dynaquant_b200 as dq
    p = dq.Propagator(N, m=M, n_traj=B, dt=DT, noise=dq.NOISE_OU if noise else dq.NOISE_NONE, seed=SEED,
                      dot=dq.DOT_HERMITIAN, precision=precision, max_steps=T)
    p.set_system(s)
    if scale_c is not None:
        p.set_coupling_classes(np.zeros(len(s.cls_off), dtype=np.int32), [scale_c])
    if noise:
        p.set_noise_params(np.full(N, SIGMA), np.full(N, TAU))
    p.set_static_energies(eps0)
    p.set_initial_state(psi0)
    p.adjoint_setup(T, LEN, 1.0 / LEN, target, checkpoint_every=ck)
    return p


def _oracle(oracle, s, eps0, psi0, target, scale_c=1.0, noise=True):
    O = oracle
    rp, col, val, _ = s.off_diagonal()
    kw = dict(noise=O.NOISE_OU, sigma=np.full(N, SIGMA), tau=np.full(N, TAU)) if noise else {}
    return O.spectrum_loss_grad(rp, col, val, s.cls_off, [scale_c], eps0, M, DT, psi0, B, T, LEN, 1.0 / LEN,
                                target, seed=SEED, **kw)


@pytest.mark.parametrize("noise,tiling", [(True, None), (False, None), (True, (8, 1, 2, 2, 2, 1)),
                                          (True, (8, 1, 1, 2, 8, 1))])
def test_adjoint_fp64_matches_oracle(oracle, noise, tiling):
    import dynaquant_b200 as dq
    s, eps0, psi0, target = _problem()
    p = _prop(dq.PREC_FP64, s, eps0, psi0, target, noise=noise)
    if tiling:   # one-kernel Lanczos iterations in both the forward and the adjoint Lanczos
        p.set_tiling(*tiling)
    loss = p.forward()
    gs, gc = p.backward()
    lo, go = _oracle(oracle, s, eps0, psi0, target, noise=noise)
    assert loss == pytest.approx(lo, rel=1e-10)
    scale = np.abs(go[:N]).max()
    assert np.abs(gs - go[:N]).max() <= GRAD_TOL_FP64 * scale
    assert gc[0] == pytest.approx(go[N], rel=GRAD_TOL_FP64)
    p.close()


def test_adjoint_class_scale_and_checkpointing(oracle):
    import dynaquant_b200 as dq
    s, eps0, psi0, target = _problem()
    p = _prop(dq.PREC_FP64, s, eps0, psi0, target, scale_c=1.3)
    loss_a = p.forward()
    ga, gca = p.backward()
    lo, go = _oracle(oracle, s, eps0, psi0, target, scale_c=1.3)
    assert loss_a == pytest.approx(lo, rel=1e-10)
    assert np.abs(ga - go[:N]).max() <= GRAD_TOL_FP64 * np.abs(go[:N]).max()
    assert gca[0] == pytest.approx(go[N], rel=GRAD_TOL_FP64)
    # segments of 5 steps recomputed from checkpoints give the same numbers
    q = _prop(dq.PREC_FP64, s, eps0, psi0, target, scale_c=1.3, ck=5)
    loss_b = q.forward()
    gb, gcb = q.backward()
    assert loss_b == loss_a
    assert np.abs(gb - ga).max() <= 1e-13 * np.abs(ga).max()
    assert gcb[0] == pytest.approx(gca[0], rel=1e-13)
    # a second forward/backward on the same context repeats itself
    assert q.forward() == loss_b
    gb2, _ = q.backward()
    assert np.array_equal(gb2, gb)
    p.close()
    q.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_adjoint_two_classes_matches_oracle(oracle, precision):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    _, eps0, psi0, target = _problem()
    lat = systems.lattice2d(8, seed=2)            # 64 sites, nearest (class 0) and next-nearest (class 1)
    scales = [1.1, 0.9]
    p = dq.Propagator(N, m=M, n_traj=B, dt=DT, noise=dq.NOISE_OU, seed=SEED, dot=dq.DOT_HERMITIAN,
                      precision=dq.PREC_FP64 if precision == "fp64" else dq.PREC_MIXED, max_steps=T)
    p.set_system(lat)
    p.set_coupling_classes(lat.cls_off, scales)
    p.set_noise_params(np.full(N, SIGMA), np.full(N, TAU))
    p.set_static_energies(eps0)
    p.set_initial_state(psi0)
    p.adjoint_setup(T, LEN, 1.0 / LEN, target)
    loss = p.forward()
    gs, gc = p.backward()
    O = oracle
    rp, col, val, _ = lat.off_diagonal()
    lo, go = O.spectrum_loss_grad(rp, col, val, lat.cls_off, scales, eps0, M, DT, psi0, B, T, LEN, 1.0 / LEN,
                                  target, seed=SEED, noise=O.NOISE_OU, sigma=np.full(N, SIGMA),
                                  tau=np.full(N, TAU))
    tol = GRAD_TOL_FP64 if precision == "fp64" else GRAD_TOL_MIXED
    assert loss == pytest.approx(lo, rel=1e-10 if precision == "fp64" else 1e-5)
    assert np.abs(gs - go[:N]).max() <= tol * np.abs(go[:N]).max()
    assert np.allclose(gc, go[N:], rtol=tol, atol=tol * np.abs(go[N:]).max())
    p.close()


def test_adjoint_fd_on_gpu():
    import dynaquant_b200 as dq
    s, eps0, psi0, target = _problem()
    p = _prop(dq.PREC_FP64, s, eps0, psi0, target)
    p.forward()
    g, _ = p.backward()
    h = 1e-3
    for i in (27, 31, 36):   # sites the wavepacket reaches within the run
        e1, e2 = eps0.copy(), eps0.copy()
        e1[i] += h
        e2[i] -= h
        p.set_static_energies(e1)
        f1 = p.forward()
        p.set_static_energies(e2)
        f2 = p.forward()
        fd = (f1 - f2) / (2 * h)
        assert abs(g[i] - fd) <= FD_TOL * abs(fd), (i, g[i], fd)
    p.close()


def test_adjoint_mixed_matches_oracle(oracle):
    import dynaquant_b200 as dq
    s, eps0, psi0, target = _problem()
    p = _prop(dq.PREC_MIXED, s, eps0, psi0, target)
    loss = p.forward()
    gs, gc = p.backward()
    lo, go = _oracle(oracle, s, eps0, psi0, target)
    assert loss == pytest.approx(lo, rel=1e-5)
    assert np.abs(gs - go[:N]).max() <= GRAD_TOL_MIXED * np.abs(go[:N]).max()
    assert gc[0] == pytest.approx(go[N], rel=GRAD_TOL_MIXED)
    p.close()


def test_adjoint_rejects_bad_use():
    import dynaquant_b200 as dq
    s, eps0, psi0, target = _problem()
    p = dq.Propagator(N, m=M, n_traj=B, dt=DT, dot=dq.DOT_BILINEAR, precision=dq.PREC_FP64, max_steps=T)
    p.set_system(s)
    p.set_initial_state(psi0)
    with pytest.raises(dq.DQError, match="Hermitian"):
        p.adjoint_setup(T, LEN, 1.0, target)
    p.close()
    q = _prop(dq.PREC_FP64, s, eps0, psi0, target)
    with pytest.raises(dq.DQError, match="forward"):
        q.backward()
    with pytest.raises(dq.DQError, match="fft_len"):
        q.adjoint_setup(T, 8, 1.0, target[:8])
    q.close()
