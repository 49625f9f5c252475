"""Generates the golden fixtures in tests/golden/ with the CPU oracle.

The reference's own trajectories cannot be regenerated (its seeds come from
the wall clock, systemClass.cu:767/890-891/1012, and its Hamiltonian file
data-example/hamInner.dat is not distributed), so trajectory-level goldens are
produced by the oracle with fixed Philox seeds on the reduced chain
workload (1-D chain, N = 1024, J = -300 cm^-1, static disorder 100 cm^-1, OU
noise 200 cm^-1 / 100 fs, dt = 1 fs, m = 16, psi0 on site 512), 4
trajectories x 60 steps.  Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from dynaquant_b200 import systems  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

CHAIN = dict(n=1024, J=-300.0, m=16, dt=1.0, sigma=200.0, tau=100.0, sigma_static=100.0, seed=20240611,
             n_traj=4, n_steps=60, pop_every=10, init_site=512)


def chain_system(dot_mode):
    s = systems.chain(CHAIN["n"], CHAIN["J"])
    rp, col, val, diag = s.off_diagonal()
    return O.System(rp, col, val, diag, m=CHAIN["m"], dt=CHAIN["dt"], dot_mode=dot_mode, noise=O.NOISE_OU,
                    sigma=CHAIN["sigma"], tau=CHAIN["tau"], sigma_static=CHAIN["sigma_static"], seed=CHAIN["seed"])


def chain_psi0():
    psi0 = np.zeros(CHAIN["n"], dtype=np.complex128)
    psi0[CHAIN["init_site"]] = 1.0
    return psi0


def make():
    O.build()
    out = {}
    for dot, tag in ((O.DOT_HERMITIAN, "herm"), (O.DOT_BILINEAR, "bil")):
        S = chain_system(dot)
        r = S.run(CHAIN["n_traj"], CHAIN["n_steps"], chain_psi0(), pop_every=CHAIN["pop_every"], threads=1,
                  want_final=True)
        out[f"{tag}_pops"] = r["pops"]
        out[f"{tag}_corr"] = r["corr"]
        out[f"{tag}_err"] = r["err"]
        if tag == "herm":
            out[f"{tag}_psi_final"] = r["psi_final"]
    # noise state of trajectory 1 after 60 OU updates
    S = chain_system(O.DOT_HERMITIAN)
    eps, deps = S.traj_init(1)
    for k in range(CHAIN["n_steps"]):
        S.noise_update(1, k, eps, deps)
    out["noise_traj1_eps"] = eps
    out["noise_traj1_deps"] = deps
    # normals for a few keys (bitwise pin of the Philox + Box-Muller chain)
    keys = np.array([[7, 1, 3, 5, 11, s] for s in range(6)] + [[2 ** 40 + 9, 2, 0, 99, 123456, 0]], dtype=np.uint64)
    out["normal_keys"] = keys
    out["normal_vals"] = np.array([O.normal(int(k[0]), int(k[1]), int(k[2]), int(k[3]), int(k[4]), int(k[5]))
                                   for k in keys])
    # Padé exponential of a fixed augmented matrix
    rng = np.random.default_rng(5)
    m = 12
    al = np.zeros(m + 2, complex)
    be = np.zeros(m + 2, complex)
    al[1:m + 1] = rng.normal(0, 300, m)
    be[1:m + 1] = np.abs(rng.normal(300, 50, m))
    T = np.zeros((m + 2, m + 2), complex)
    for i in range(m):
        T[i, i] = al[i + 1]
        if i + 1 < m:
            T[i, i + 1] = T[i + 1, i] = be[i + 1]
    T[0, m] = 1.0
    T[m, m + 1] = 1.0
    A = (-1j * 1.0 / O.hbar_reference()) * T
    E, s = O.pade_exp(A, O.NORM_COMPLEX)
    out["pade_A"] = A
    out["pade_E"] = E
    np.savez_compressed(os.path.join(HERE, "golden_chain.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_chain.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    make()
