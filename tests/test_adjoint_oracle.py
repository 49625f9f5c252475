"""CPU checks of the oracle's spectrum-loss adjoint: the loss agrees with the forward ensemble run,
and the hand-derived gradient agrees with central finite differences of the loss."""
import numpy as np
import pytest

from dynaquant_b200 import systems


def _problem(O, noise):
    S = systems.lattice2d(6, seed=3)
    rp, col, val, _ = S.off_diagonal()
    rng = np.random.default_rng(1)
    eps0 = rng.normal(0.0, 100.0, S.n)
    length = 64
    kw = dict(m=14, dt=2.0, psi0=S.bright_state((1.0, 0.0, 0.0)), n_traj=2, n_steps=24, length=length,
              scale=1.0 / length, target=rng.normal(0.0, 0.05, length), noise=noise,
              sigma=np.full(S.n, 60.0), tau=np.full(S.n, 80.0), seed=7)
    return S, rp, col, val, eps0, kw


def test_loss_matches_forward_run(oracle):
    O = oracle
    S, rp, col, val, eps0, kw = _problem(O, O.NOISE_OU)
    loss, _ = O.spectrum_loss_grad(rp, col, val, S.cls_off, [1.0, 1.0], eps0, want_grad=False, **kw)
    sysm = O.System(rp, col, val, eps0, kw["m"], kw["dt"], dot_mode=O.DOT_HERMITIAN, norm_mode=O.NORM_COMPLEX,
                    noise=O.NOISE_OU, sigma=kw["sigma"], tau=kw["tau"], static_eps=eps0, seed=kw["seed"])
    r = sysm.run(kw["n_traj"], kw["n_steps"], kw["psi0"])
    spec = np.zeros(kw["length"], dtype=np.complex128)
    spec[: kw["n_steps"] + 1] = r["corr"]
    A = kw["scale"] * np.real(np.fft.ifft(spec) * kw["length"])
    assert loss == pytest.approx(float(np.sum((A - kw["target"]) ** 2)), rel=1e-12)


@pytest.mark.parametrize("noise", ["none", "ou"])
def test_gradient_matches_finite_differences(oracle, noise):
    O = oracle
    S, rp, col, val, eps0, kw = _problem(O, O.NOISE_OU if noise == "ou" else O.NOISE_NONE)
    cls, scales = S.cls_off, np.array([1.0, 1.0])
    _, g = O.spectrum_loss_grad(rp, col, val, cls, scales, eps0, **kw)

    def f(eps, sc):
        return O.spectrum_loss_grad(rp, col, val, cls, sc, eps, want_grad=False, **kw)[0]

    h = 1e-3  # cm^-1 on energies of ~100 cm^-1
    for i in (0, 7, 20, 35):
        e1, e2 = eps0.copy(), eps0.copy()
        e1[i] += h
        e2[i] -= h
        fd = (f(e1, scales) - f(e2, scales)) / (2 * h)
        assert abs(g[i] - fd) <= 1e-5 * abs(fd), (i, g[i], fd)
    for c in range(2):
        s1, s2 = scales.copy(), scales.copy()
        s1[c] += 1e-5
        s2[c] -= 1e-5
        fd = (f(eps0, s1) - f(eps0, s2)) / 2e-5
        assert abs(g[S.n + c] - fd) <= 1e-5 * abs(fd), (c, g[S.n + c], fd)
