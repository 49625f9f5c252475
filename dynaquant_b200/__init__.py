"""dynaquant_b200 — B200 (sm_100a) stochastic-Hamiltonian exciton propagator.

Python front end of the C ABI in include/dq.h (libdq.so, built in-tree by
dynaquant_b200/build.py).  The names follow the reference's step sequence
(propagate.cu:211-254): ``prop_step`` is lanczosClass::doLanczos +
padeClass::doPade + propagateSystem + renormalizeAndStoreNorm for one
trajectory; ``run`` is the ensemble loop over all trajectories.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (DOT_BILINEAR, DOT_HERMITIAN, NOISE_GAUSS, NOISE_NONE, NOISE_OU, NOISE_ZZ, NORM_COMPLEX,
                   NORM_REAL_ONLY, PREC_FP64, PREC_MIXED, DQError)

__all__ = ["Propagator", "Group", "DQError", "NOISE_NONE", "NOISE_GAUSS", "NOISE_OU", "NOISE_ZZ", "DOT_BILINEAR", "DOT_HERMITIAN",
           "NORM_REAL_ONLY", "NORM_COMPLEX", "PREC_FP64", "PREC_MIXED", "reference_hbar"]


def reference_hbar() -> float:
    """hbar in cm^-1 fs as cppUtility.cpp:19-22 computes it (c = 299792548 m/s)."""
    import math
    return (1 / 100.) * 1e15 * 1. / (299792548. * 2 * (math.atan(1.0) * 4.0))


class Propagator:
    """One context of the C ABI: a system, its trajectories and observables.

    `device` is the CUDA ordinal the context lives on; every call runs there and
    leaves the caller's current device as it was."""

    def __init__(self, n_sites, m=16, n_traj=1, dt=1.0, hbar=0.0, noise=NOISE_NONE, ka_substeps=1,
                 sigma_static=0.0, seed=0, dot=DOT_HERMITIAN, norm=NORM_COMPLEX, precision=PREC_MIXED,
                 reorth=0, pop_every=1, max_steps=1024, device=0, m_min=0, m_tol=0.0):
        self.L = _lib.load()
        cfg = _lib.Config()
        self.L.dq_config_default(C.byref(cfg))
        cfg.n_sites, cfg.m, cfg.n_traj, cfg.dt, cfg.hbar = n_sites, m, n_traj, dt, hbar
        cfg.noise_model, cfg.ka_substeps, cfg.sigma_static, cfg.seed = noise, ka_substeps, sigma_static, seed
        cfg.dot_mode, cfg.norm_mode, cfg.precision, cfg.reorth = dot, norm, precision, reorth
        cfg.pop_every, cfg.max_steps, cfg.device = pop_every, max_steps, device
        cfg.m_min, cfg.m_tol = m_min, m_tol
        self.cfg = cfg
        self.n = n_sites
        self.n_traj = n_traj
        self.ipr_enabled = False
        h = C.c_void_p()
        rc = self.L.dq_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise DQError(rc, "dq_create failed (bad config or CUDA unavailable)")
        self.h = h

    # -- lifecycle -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.dq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise DQError(rc, self.L.dq_last_error(self.h).decode(errors="replace"))

    @property
    def stream(self) -> int:
        return self.L.dq_get_stream(self.h)

    # -- system ----------------------------------------------------------------
    def set_hamiltonian_csr(self, rowptr, col, val):
        self._rp = np.ascontiguousarray(rowptr, dtype=np.int32)
        self._col = np.ascontiguousarray(col, dtype=np.int32)
        self._val = np.ascontiguousarray(val, dtype=np.float64)
        self._check(self.L.dq_set_hamiltonian_csr(self.h, self.n, _lib.iptr(self._rp), _lib.iptr(self._col),
                                                  _lib.dptr(self._val)))

    def set_system(self, system):
        self.set_hamiltonian_csr(system.rowptr, system.col, system.val)

    def set_coupling_classes(self, cls, scales):
        cls = np.ascontiguousarray(cls, dtype=np.int32)
        scales = np.ascontiguousarray(scales, dtype=np.float64)
        self._check(self.L.dq_set_coupling_classes(self.h, _lib.iptr(cls), len(scales), _lib.dptr(scales)))
        self._n_classes = len(scales)

    def set_noise_params(self, sigma, tau=None):
        sigma = np.ascontiguousarray(np.broadcast_to(sigma, (self.n,)), dtype=np.float64)
        tau = None if tau is None else np.ascontiguousarray(np.broadcast_to(tau, (self.n,)), dtype=np.float64)
        self._check(self.L.dq_set_noise_params(self.h, _lib.dptr(sigma), _lib.dptr(tau)))

    def set_zz_spectral_density(self, omega, J, d_omega, temperature):
        """Spectral density of the ZZ real noise: omega and J in cm^-1 at spacing d_omega, temperature in K."""
        omega = np.ascontiguousarray(omega, dtype=np.float64)
        J = np.ascontiguousarray(J, dtype=np.float64)
        if omega.shape != J.shape or omega.ndim != 1:
            raise ValueError("omega and J must be 1-D arrays of one length")
        self._check(self.L.dq_set_zz_spectral_density(self.h, len(omega), _lib.dptr(omega), _lib.dptr(J),
                                                      float(d_omega), float(temperature)))

    def set_static_energies(self, eps):
        eps = None if eps is None else np.ascontiguousarray(eps, dtype=np.float64)
        self._check(self.L.dq_set_static_energies(self.h, _lib.dptr(eps)))

    def set_initial_state(self, psi0):
        psi0 = np.ascontiguousarray(psi0, dtype=np.complex128)
        self._check(self.L.dq_set_initial_state(self.h, _lib.dptr(psi0.view(np.float64))))

    def set_initial_dipole(self, mu):
        """psi0 = mu / |mu| from one direction's transition dipoles (absorption)."""
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        self._check(self.L.dq_set_initial_dipole(self.h, _lib.dptr(mu)))

    def reset(self):
        self._check(self.L.dq_reset(self.h))

    # -- propagation -------------------------------------------------------------
    def prop_step(self, traj, step, psi_in_ptr, psi_out_ptr, want_error=False):
        """One plain FP64 step on device buffers (raw CUDA pointers, N complex128)."""
        err = C.c_double()
        self._check(self.L.dq_prop_step(self.h, traj, step, C.c_void_p(psi_in_ptr), C.c_void_p(psi_out_ptr),
                                        C.byref(err) if want_error else None))
        return err.value if want_error else None

    def run_plain(self, n_steps):
        self._check(self.L.dq_run_plain(self.h, n_steps))

    def run(self, n_steps):
        self._check(self.L.dq_run(self.h, n_steps))

    def set_tiling(self, traj_chunk, vec, ctas_per_sm, rows_per_block=4, staged=0, groups=1):
        self._check(self.L.dq_set_tiling(self.h, traj_chunk, vec, ctas_per_sm, rows_per_block, staged, groups))

    def get_tiling(self):
        v = [C.c_int() for _ in range(6)]
        self._check(self.L.dq_get_tiling(self.h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def time_iteration(self, reps=10):
        """Mean device ms of one Lanczos iteration (SpMM + axpy) under the current tiling."""
        ms = C.c_double()
        self._check(self.L.dq_time_iteration(self.h, reps, C.byref(ms)))
        return ms.value

    def time_gather_floor(self, reps=10):
        """Mean device ms of the gathers alone of the current tiling's packed coupling blocks (complex64,
        vec 2, rows_per_block <= 3): the floor under the L1-gather SpMM."""
        ms = C.c_double()
        self._check(self.L.dq_time_gather_floor(self.h, reps, C.byref(ms)))
        return ms.value

    def debug_set_wait_cycles(self, cycles):
        """Test hook: budget of the TMA-fed SpMM forms' barrier waits on this device (0: default; negative:
        the ring form's CTAs first wait that many cycles on a barrier nothing completes, so they time out)."""
        self._check(self.L.dq_debug_set_wait_cycles(self.h, int(cycles)))

    def autotune_raw(self, reps=5):
        ms = C.c_double()
        self._check(self.L.dq_autotune(self.h, reps, C.byref(ms)))
        return ms.value

    def autotune(self, reps=5, use_cache=True):
        """Picks the ensemble tiling (JSON-cached per GPU and size class)."""
        from . import autotune as _at
        nnz = int(self._rp[-1]) if getattr(self, "_rp", None) is not None else 0
        return _at.tune(self, nnz, reps=reps, use_cache=use_cache)

    def profile_step(self, n_steps=1):
        """Eager steps with CUDA events between kernels: {kind: (ms per launch, launches)}."""
        nk = len(_lib.KIND_NAMES)
        ms = np.zeros(nk)
        cnt = np.zeros(nk, dtype=np.int32)
        self._check(self.L.dq_profile_step(self.h, n_steps, _lib.dptr(ms), _lib.iptr(cnt), nk))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.KIND_NAMES)}

    # -- observables -------------------------------------------------------------
    def populations(self) -> np.ndarray:
        nrec = C.c_int()
        self._check(self.L.dq_get_populations(self.h, None, C.byref(nrec)))
        out = np.zeros((nrec.value, self.n))
        self._check(self.L.dq_get_populations(self.h, _lib.dptr(out), C.byref(nrec)))
        return out

    def correlation(self) -> np.ndarray:
        npts = C.c_int()
        self._check(self.L.dq_get_correlation(self.h, None, C.byref(npts)))
        out = np.zeros(npts.value, dtype=np.complex128)
        self._check(self.L.dq_get_correlation(self.h, _lib.dptr(out.view(np.float64)), C.byref(npts)))
        return out

    def states(self) -> np.ndarray:
        out = np.zeros((self.n_traj, self.n), dtype=np.complex128)
        self._check(self.L.dq_get_states(self.h, _lib.dptr(out.view(np.float64))))
        return out

    def error_accum(self) -> np.ndarray:
        out = np.zeros(self.n_traj)
        self._check(self.L.dq_get_error_accum(self.h, _lib.dptr(out)))
        return out

    def spectrum(self, length) -> np.ndarray:
        out = np.zeros(length, dtype=np.complex128)
        self._check(self.L.dq_get_spectrum(self.h, length, _lib.dptr(out.view(np.float64))))
        return out

    def noise_state(self, traj):
        eps = np.zeros(self.n)
        deps = np.zeros(self.n)
        self._check(self.L.dq_get_noise_state(self.h, traj, _lib.dptr(eps), _lib.dptr(deps)))
        return eps, deps

    # -- the reference's output files ---------------------------------------------
    def write_populations(self, path, binary=False, continuation=False):
        """pops.dat (popPrintClass format): population sums over trajectories per recorded step."""
        self._check(self.L.dq_write_populations(self.h, str(path).encode(), int(binary), int(continuation)))

    def write_states(self, folder):
        """folder/_states_<t>.dat (statePrintClass format) for the current step."""
        self._check(self.L.dq_write_states(self.h, str(folder).encode()))

    def write_spectrum(self, corr_path, spec_path, scaling=1.0):
        """Correlation and spectrum text files (spectraClass format), transform length steps + 1."""
        self._check(self.L.dq_write_spectrum(self.h, str(corr_path).encode(), str(spec_path).encode(),
                                             float(scaling)))

    def set_line_dressing(self, sigma_fs):
        """Gaussian line-shape dressing of the correlation before transforms (0 turns it off)."""
        self._check(self.L.dq_set_line_dressing(self.h, float(sigma_fs)))

    def write_ipr(self, path):
        """invParticRat.dat: the ensemble-mean inverse participation ratio of steps 0..steps-1."""
        self._check(self.L.dq_write_ipr(self.h, str(path).encode()))

    # -- Taylor-Krylov mode and the inverse participation ratio ---------------------
    def set_taylor_krylov(self, p, m_b=None, rowptr=None, col=None, val=None):
        """Taylor-Krylov propagation of order p with m_b Lanczos iterations on the auxiliary matrix B
        (full CSR over the sites, diagonal included); p = 0 returns to Lanczos mode."""
        if p == 0:
            self._check(self.L.dq_set_taylor_krylov(self.h, 0, 0, None, None, None))
            return
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        self._check(self.L.dq_set_taylor_krylov(self.h, int(p), int(m_b), _lib.iptr(rowptr), _lib.iptr(col),
                                                _lib.dptr(val)))

    def set_correlation_bra(self, bra):
        """Bra of the correlation M(t) = <bra|psi(t)> (CD spectra); None returns to psi0."""
        if bra is None:
            self._check(self.L.dq_set_correlation_bra(self.h, None))
            return
        bra = np.ascontiguousarray(bra, dtype=np.complex128)
        self._check(self.L.dq_set_correlation_bra(self.h, _lib.dptr(bra.view(np.float64))))

    # -- sharded ensembles ------------------------------------------------------------
    def set_trajectory_offset(self, traj0):
        """Index of this context's trajectory 0 in the whole ensemble (even): the random-draw key."""
        self._check(self.L.dq_set_trajectory_offset(self.h, int(traj0)))

    def observable_sums(self, with_ipr=False):
        """Raw sums over this context's trajectories: (pops, corr, ipr or None)."""
        T = self.steps_done
        pops = np.zeros((T // self.cfg.pop_every + 1, self.n))
        corr = np.zeros(T + 1, dtype=np.complex128)
        ipr = np.zeros(T + 1) if with_ipr else None
        self._check(self.L.dq_get_observable_sums(self.h, _lib.dptr(pops), _lib.dptr(corr.view(np.float64)),
                                                  _lib.dptr(ipr)))
        return pops, corr, ipr

    def set_observable_sums(self, pops, corr, ipr, n_traj_total):
        """Install observable sums reduced over all shards, standing for n_traj_total trajectories."""
        pops = np.ascontiguousarray(pops, dtype=np.float64)
        corr = np.ascontiguousarray(corr, dtype=np.complex128)
        ipr = None if ipr is None else np.ascontiguousarray(ipr, dtype=np.float64)
        self._check(self.L.dq_set_observable_sums(self.h, _lib.dptr(pops), _lib.dptr(corr.view(np.float64)),
                                                  _lib.dptr(ipr), int(n_traj_total)))

    def set_ipr(self, enable=True):
        self._check(self.L.dq_set_ipr(self.h, int(bool(enable))))
        self.ipr_enabled = bool(enable)

    def ipr(self):
        """Ensemble mean of 1 / sum_i |psi_i|^4 after 0..steps_done steps."""
        nv = C.c_int()
        self._check(self.L.dq_get_ipr(self.h, None, C.byref(nv)))
        out = np.zeros(nv.value)
        self._check(self.L.dq_get_ipr(self.h, _lib.dptr(out), C.byref(nv)))
        return out

    # -- adjoint -------------------------------------------------------------------
    def adjoint_setup(self, n_steps, fft_len, scale, target, checkpoint_every=0):
        """Fixes the spectrum-fitting loss sum_j (scale*Re(S_j) - target_j)^2 (S: inverse DFT of the
        ensemble-mean correlation over n_steps, zero-padded to fft_len) for forward()/backward()."""
        self._target = np.ascontiguousarray(target, dtype=np.float64)
        if self._target.shape != (fft_len,):
            raise ValueError("target must hold fft_len values")
        self._check(self.L.dq_adjoint_setup(self.h, n_steps, fft_len, float(scale), _lib.dptr(self._target),
                                            checkpoint_every))
        self._adj_T = int(n_steps)

    def forward(self) -> float:
        loss = C.c_double()
        self._check(self.L.dq_forward(self.h, C.byref(loss)))
        return loss.value

    def forward_shard(self):
        """Forward run of this shard; returns its raw correlation sums (steps + 1) for the all-reduce."""
        corr = np.zeros(self._adj_T + 1, dtype=np.complex128)
        self._check(self.L.dq_forward_shard(self.h, _lib.dptr(corr.view(np.float64))))
        return corr

    def forward_reduced(self, corr_sums, n_traj_total) -> float:
        """Loss of the whole ensemble from the correlation sums of all shards; prepares backward()."""
        corr = np.ascontiguousarray(corr_sums, dtype=np.complex128)
        loss = C.c_double()
        self._check(self.L.dq_forward_reduced(self.h, _lib.dptr(corr.view(np.float64)), int(n_traj_total),
                                              C.byref(loss)))
        return loss.value

    def backward(self):
        """Returns (dL/d site energies (N,), dL/d coupling-class scales (n_classes,), one entry for
        the implicit class when none were set)."""
        gs = np.zeros(self.n)
        gc = np.zeros(getattr(self, "_n_classes", 1))
        self._check(self.L.dq_backward(self.h, _lib.dptr(gs), _lib.dptr(gc)))
        return gs, gc

    @property
    def steps_done(self) -> int:
        return self.L.dq_steps_done(self.h)


class Group:
    """Several Propagators (aggregates of any size and trajectory count, one device) advanced together:
    each step is one CUDA graph with a concurrent branch per member (dq_group_*)."""

    def __init__(self, members):
        self.members = list(members)
        self.L = _lib.load()
        arr = (C.c_void_p * len(self.members))(*[m.h for m in self.members])
        h = C.c_void_p()
        rc = self.L.dq_group_create(arr, len(self.members), C.byref(h))
        if rc != 0:
            raise DQError(rc, "dq_group_create failed (members on one device, each once)")
        self.h = h

    def run(self, n_steps):
        rc = self.L.dq_group_run(self.h, n_steps)
        if rc != 0:
            raise DQError(rc, self.L.dq_group_last_error(self.h).decode(errors="replace"))

    def run_timed(self, n_steps) -> float:
        """run() returning the device milliseconds of the step launches (graph capture excluded)."""
        ms = C.c_double()
        rc = self.L.dq_group_run_timed(self.h, n_steps, C.byref(ms))
        if rc != 0:
            raise DQError(rc, self.L.dq_group_last_error(self.h).decode(errors="replace"))
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            self.L.dq_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
