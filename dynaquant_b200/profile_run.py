"""Small driver for ncu captures of the ensemble kernels.

Runs the benchmark workload (30,000-site dipole tube, 256 trajectories,
m = 20, complex64) for a few steps with a fixed tiling, no autotuning and no
CPU oracle, so a capture sees only the propagator's own launches:

    python -m dynaquant_b200.profile_run --steps 2 [--tiling 32,2,4] [--B 256] [--zz 253]
    python -m dynaquant_b200.profile_run --around 120 --along 1000 --cutoff 40 --m 24 --B 128

(the second line: the 120,000-site tube of the large workload, with fewer trajectories).

--zz N swaps the OU noise for the ZZ model with N oscillators of an Ohmic
spectral density on a 8.1357 cm^-1 grid at 77 K.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--B", type=int, default=256)
    ap.add_argument("--around", type=int, default=60)
    ap.add_argument("--along", type=int, default=500)
    ap.add_argument("--cutoff", type=float, default=25.0)
    ap.add_argument("--m", type=int, default=20)
    ap.add_argument("--tiling", default="")
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--zz", type=int, default=0)
    args = ap.parse_args()
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    s = systems.tube(args.around, args.along, cutoff=args.cutoff)
    p = dq.Propagator(s.n, m=args.m, n_traj=args.B, dt=0.5, noise=dq.NOISE_ZZ if args.zz else dq.NOISE_OU,
                      sigma_static=150.0, seed=2024, dot=dq.DOT_HERMITIAN,
                      precision=dq.PREC_FP64 if args.fp64 else dq.PREC_MIXED, pop_every=16,
                      max_steps=args.steps + 4)
    p.set_system(s)
    if args.zz:
        om = 8.1357 * np.arange(1, args.zz + 1)
        p.set_zz_spectral_density(om, 60.0 * (om / 120.0) * np.exp(-om / 120.0), 8.1357, 77.0)
    else:
        p.set_noise_params(np.full(s.n, 250.0), np.full(s.n, 50.0))
    p.set_initial_state(s.bright_state())
    if args.tiling:
        p.set_tiling(*[int(x) for x in args.tiling.split(",")])
    p.reset()
    p.run(args.steps)
    print("steps", p.steps_done, "tiling", p.get_tiling(), "pop sum", float(p.populations()[-1].sum()))
    p.close()


if __name__ == "__main__":
    main()
