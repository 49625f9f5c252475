"""Population parity at the benchmark configurations' own lengths.

Chain (1,024 sites, 64 trajectories, 1,000 steps, m = 16): the plain FP64
per-trajectory path and the batched FP64 ensemble against the FP64 oracle,
populations and correlation to 1e-10 (the step loop of propagate.cu:199-259
for every trajectory).

Tube 60 x 500 (30,000 sites, 256 trajectories, 4,096 steps, m = 20): the
mixed-precision ensemble (complex64 vectors, FP64 Lanczos scalars and Padé)
against the batched FP64 ensemble on every trajectory, populations to 1e-6
absolute and the error relative to the largest population reported per
record; and both against the oracle on 4 trajectories over 512 steps.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POP_TOL_FP64 = 1e-10
POP_TOL_MIXED = 1e-6
# largest |p_mixed - p_fp64| / max p over the 4096 steps; measured about 1e-5
# (FP32 rounding of the Krylov vectors, accumulated over the run)
REL_TOL_MIXED = 1e-3

CHAIN = dict(n=1024, J=-300.0, sigma_static=100.0, sigma=200.0, tau=100.0, dt=1.0, steps=1000, m=16,
             n_traj=64, pop_every=10, seed=101)
TUBE = dict(around=60, along=500, cutoff=25.0, sigma_static=150.0, sigma=250.0, tau=50.0, dt=0.5, steps=4096,
            m=20, n_traj=256, pop_every=16, seed=2024)


def _threads():
    return os.cpu_count() or 1


def _chain_oracle(oracle, s, c):
    rp, col, val, diag = s.off_diagonal()
    return oracle.System(rp, col, val, diag, m=c["m"], dt=c["dt"], dot_mode=oracle.DOT_HERMITIAN,
                         noise=oracle.NOISE_OU, sigma=c["sigma"], tau=c["tau"], sigma_static=c["sigma_static"],
                         seed=c["seed"])


def _prop(s, c, precision, n_traj=None, steps=None):
    import dynaquant_b200 as dq
    p = dq.Propagator(s.n, m=c["m"], n_traj=n_traj or c["n_traj"], dt=c["dt"], noise=dq.NOISE_OU,
                      sigma_static=c["sigma_static"], seed=c["seed"], dot=dq.DOT_HERMITIAN, precision=precision,
                      pop_every=c["pop_every"], max_steps=steps or c["steps"])
    p.set_system(s)
    p.set_noise_params(np.full(s.n, c["sigma"]), np.full(s.n, c["tau"]))
    return p


def test_chain_1000_steps_plain_and_ensemble_fp64_match_oracle(oracle):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    c = CHAIN
    s = systems.chain(c["n"], c["J"])
    psi0 = np.zeros(c["n"], complex)
    psi0[512] = 1.0
    ref = _chain_oracle(oracle, s, c).run(c["n_traj"], c["steps"], psi0, pop_every=c["pop_every"],
                                          threads=_threads())
    p = _prop(s, c, dq.PREC_FP64)
    p.set_initial_state(psi0)
    p.run_plain(c["steps"])
    d_pops = np.abs(p.populations() - ref["pops"]).max()
    d_corr = np.abs(p.correlation() - ref["corr"]).max()
    print(f"chain plain FP64, {c['n_traj']} traj x {c['steps']} steps: max|dp| {d_pops:.3e}, max|dC| {d_corr:.3e}")
    assert d_pops < POP_TOL_FP64 and d_corr < POP_TOL_FP64
    assert np.allclose(p.error_accum(), ref["err"], rtol=1e-3, atol=1e-13)
    p.reset()
    p.run(c["steps"])
    d_pops = np.abs(p.populations() - ref["pops"]).max()
    d_corr = np.abs(p.correlation() - ref["corr"]).max()
    print(f"chain ensemble FP64: max|dp| {d_pops:.3e}, max|dC| {d_corr:.3e}")
    assert d_pops < POP_TOL_FP64 and d_corr < POP_TOL_FP64
    p.close()


def _tube():
    from dynaquant_b200 import systems
    t = TUBE
    return systems.tube(t["around"], t["along"], cutoff=t["cutoff"])


def test_tube_4096_steps_mixed_against_fp64_ensemble():
    import dynaquant_b200 as dq
    t = TUBE
    s = _tube()
    psi0 = s.bright_state()
    out = {}
    for prec in (dq.PREC_FP64, dq.PREC_MIXED):
        p = _prop(s, t, prec)
        p.set_initial_state(psi0)
        p.autotune()
        p.reset()
        p.run(t["steps"])
        out[prec] = (p.populations(), p.correlation())
        p.close()
    (p64, c64), (p32, c32) = out[dq.PREC_FP64], out[dq.PREC_MIXED]
    d_abs = np.abs(p32 - p64).max(axis=1)
    d_rel = d_abs / p64.max(axis=1)
    steps = np.arange(len(d_abs)) * t["pop_every"]
    for k in (1, 4, 16, 64, 128, 256):
        if k < len(d_abs):
            print(f"tube mixed vs FP64 at step {steps[k]}: max|dp| {d_abs[k]:.3e}, relative {d_rel[k]:.3e}")
    print(f"tube mixed vs FP64 over {t['steps']} steps: max|dp| {d_abs.max():.3e}, relative {d_rel.max():.3e}, "
          f"max|dC| {np.abs(c32 - c64).max():.3e}")
    assert d_abs.max() < POP_TOL_MIXED
    assert d_rel.max() < REL_TOL_MIXED
    assert np.abs(c32 - c64).max() < 1e-4


def test_tube_512_steps_both_precisions_against_oracle(oracle):
    import dynaquant_b200 as dq
    t = TUBE
    s = _tube()
    psi0 = s.bright_state()
    rp, col, val, diag = s.off_diagonal()
    S = oracle.System(rp, col, val, diag, m=t["m"], dt=t["dt"], dot_mode=oracle.DOT_HERMITIAN, noise=oracle.NOISE_OU,
                      sigma=t["sigma"], tau=t["tau"], sigma_static=t["sigma_static"], seed=t["seed"])
    B, T = 4, 512
    ref = S.run(B, T, psi0, pop_every=t["pop_every"], threads=min(B, _threads()))
    for prec, tol in ((dq.PREC_FP64, POP_TOL_FP64), (dq.PREC_MIXED, POP_TOL_MIXED)):
        p = _prop(s, t, prec, n_traj=B, steps=T)
        p.set_initial_state(psi0)
        p.run(T)
        d = np.abs(p.populations() - ref["pops"]).max(axis=1)
        rel = d / ref["pops"].max(axis=1)
        print(f"tube {'FP64' if prec == dq.PREC_FP64 else 'mixed'} vs oracle, {B} traj x {T} steps: "
              f"max|dp| {d.max():.3e}, relative {rel.max():.3e}")
        assert d.max() < tol
        p.close()
