"""Adjoint gradient at full size on the 64x64 lattice (4096 site energies + 2 coupling scales,
128 trajectories, 2000 steps, m = 16, checkpoints every 50 steps, 4096-point spectrum, OU noise
200 cm^-1 / 100 fs held fixed by common Philox seeds), FP64: the gradient of 32 random parameters
against central finite differences of the GPU forward loss (h = 1e-3 cm^-1 on site energies)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FD_REL_TOL = 1e-5


def test_lattice_gradient_matches_central_differences():
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    lat = systems.lattice2d(64, J_nn=-250.0, J_nnn=40.0, seed=0)
    n, T, L = lat.n, 2000, 4096
    eps = np.random.default_rng(0).normal(0.0, 100.0, n)
    eps_t = eps + np.random.default_rng(1).normal(0.0, 30.0, n)
    p = dq.Propagator(n, m=16, n_traj=128, dt=1.0, noise=dq.NOISE_OU, seed=77, dot=dq.DOT_HERMITIAN,
                      precision=dq.PREC_FP64, max_steps=T)
    p.set_system(lat)
    p.set_coupling_classes(lat.cls_off, [1.0, 1.0])
    p.set_noise_params(np.full(n, 200.0), np.full(n, 100.0))
    p.set_initial_state(lat.bright_state((1.0, 0.0, 0.0)))
    p.set_static_energies(eps_t)
    p.run(T)
    target = (1.0 / T) * p.spectrum(L).real
    p.set_static_energies(eps)
    p.adjoint_setup(T, L, 1.0 / T, target, checkpoint_every=50)
    p.forward()
    gs, gc = p.backward()
    rng = np.random.default_rng(2)
    sites = rng.choice(n, 30, replace=False)
    errs = []
    for i in sites:
        e1, e2 = eps.copy(), eps.copy()
        e1[i] += 1e-3
        e2[i] -= 1e-3
        p.set_static_energies(e1)
        f1 = p.forward()
        p.set_static_energies(e2)
        f2 = p.forward()
        fd = (f1 - f2) / 2e-3
        errs.append((f"eps[{i}]", gs[i], fd, abs(gs[i] - fd) / abs(fd)))
    p.set_static_energies(eps)
    for q in range(2):
        f = []
        for sgn in (1, -1):
            sc = [1.0, 1.0]
            sc[q] += sgn * 1e-5
            p.set_coupling_classes(lat.cls_off, sc)
            f.append(p.forward())
        fd = (f[0] - f[1]) / 2e-5
        errs.append((f"scale[{q}]", gc[q], fd, abs(gc[q] - fd) / abs(fd)))
    p.close()
    worst = max(errs, key=lambda e: e[3])
    assert worst[3] <= FD_REL_TOL, worst
