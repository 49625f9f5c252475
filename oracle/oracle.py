"""ctypes front end of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module as the checker; the product library
(dynaquant_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

NOISE_NONE, NOISE_GAUSS, NOISE_OU, NOISE_ZZ = 0, 1, 2, 3
DOT_BILINEAR, DOT_HERMITIAN = 0, 1
NORM_REAL_ONLY, NORM_COMPLEX = 0, 1
P_OU, P_GAUSS, P_OU_INIT, P_STATIC, P_ZZPHASE = 1, 2, 3, 4, 5


def build() -> str:
    """Compile liboracle.so with its Makefile (no-op when up to date), and, where the
    reference's sources are present, its input-line functions into _ref/."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    subprocess.run(["make", "-s", "-C", _HERE, "ref"], check=False)
    return _LIB


REF_INFILE = os.path.join(_HERE, "_ref", "libref_infile.so")


def ref_parse_line(line: str):
    """The reference's own stringSplit + stringTrim on one input line (cppUtility.cpp:82-106):
    (key, value), None for a line without '=' or a key with '!', or "throws" where the
    reference's substr would throw.  Needs _ref/libref_infile.so."""
    L = C.CDLL(REF_INFILE)
    k = C.create_string_buffer(4096)
    v = C.create_string_buffer(4096)
    rc = L.ref_parse_line(line.encode(), k, len(k), v, len(v))
    if rc == -1:
        return "throws"
    if rc != 1:
        return None
    return k.value.decode(), v.value.decode()


class _System(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("rowptr", C.POINTER(C.c_int)),
        ("col", C.POINTER(C.c_int)),
        ("val", C.POINTER(C.c_double)),
        ("h0diag", C.POINTER(C.c_double)),
        ("m", C.c_int),
        ("dt", C.c_double),
        ("hbar", C.c_double),
        ("dot_mode", C.c_int),
        ("norm_mode", C.c_int),
        ("noise", C.c_int),
        ("ka_substeps", C.c_int),
        ("sigma", C.POINTER(C.c_double)),
        ("tau", C.POINTER(C.c_double)),
        ("sigma_static", C.c_double),
        ("static_eps", C.POINTER(C.c_double)),
        ("seed", C.c_uint64),
        ("reorth", C.c_int),
        ("m_min", C.c_int),
        ("m_tol", C.c_double),
        ("n_osc", C.c_int),
        ("zz_omega", C.POINTER(C.c_double)),
        ("zz_coeff", C.POINTER(C.c_double)),
        ("tk_p", C.c_int),
        ("tk_m", C.c_int),
        ("tk_rowptr", C.POINTER(C.c_int)),
        ("tk_col", C.POINTER(C.c_int)),
        ("tk_val", C.POINTER(C.c_double)),
        ("tk_diag", C.POINTER(C.c_double)),
        ("corr_bra", C.POINTER(C.c_double)),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        dp = C.POINTER(C.c_double)
        L.dqo_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        L.dqo_log.argtypes = [C.c_double]
        L.dqo_log.restype = C.c_double
        L.dqo_sincos_2pi.argtypes = [C.c_double, dp, dp]
        L.dqo_normal.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.dqo_normal.restype = C.c_double
        L.dqo_hbar_reference.restype = C.c_double
        L.dqo_pade_ck.argtypes = [C.c_int, dp]
        L.dqo_pade_exp.argtypes = [C.c_int, dp, dp, C.c_int]
        L.dqo_pade_exp.restype = C.c_int
        sp = C.POINTER(_System)
        L.dqo_traj_init.argtypes = [sp, C.c_int, dp, dp]
        L.dqo_noise_update.argtypes = [sp, C.c_int, C.c_int, dp, dp, dp]
        L.dqo_krylov_step.argtypes = [sp, dp, dp, dp, dp, dp, C.POINTER(C.c_int)]
        L.dqo_krylov_step.restype = C.c_int
        L.dqo_krylov_step_m.argtypes = [sp, dp, dp, dp, dp, dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.dqo_krylov_step_m.restype = C.c_int
        L.dqo_lanczos.argtypes = [sp, dp, dp, dp, dp, dp]
        L.dqo_lanczos.restype = C.c_double
        L.dqo_build_tbar.argtypes = [C.c_int, dp, dp, dp]
        L.dqo_run.argtypes = [sp, C.c_int, C.c_int, C.c_int, dp, C.c_int, dp, dp, dp, dp, dp, C.c_int]
        L.dqo_tk_step.argtypes = [sp, dp, dp, dp, dp, dp]
        L.dqo_tk_step.restype = C.c_int
        L.dqo_run.restype = C.c_int
        L.dqo_ifft.argtypes = [C.c_int, dp]
        L.dqo_zz_coefficients.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, dp, dp]
        L.dqo_zz_phase.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        L.dqo_zz_phase.restype = C.c_float
        L.dqo_noise_update_zz.argtypes = [sp, C.c_int, dp, C.POINTER(C.c_float), dp]
        ip = C.POINTER(C.c_int)
        L.dqo_spectrum_loss_grad.argtypes = [sp, dp, ip, C.c_int, C.c_int, C.c_int, dp, C.c_int, C.c_double,
                                             dp, dp, C.c_int]
        L.dqo_spectrum_loss_grad.restype = C.c_double
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().dqo_philox4x32_10(c, k, o)
    return list(o)


def log(x):
    return lib().dqo_log(float(x))


def sincos_2pi(u):
    s, c = C.c_double(), C.c_double()
    lib().dqo_sincos_2pi(float(u), C.byref(s), C.byref(c))
    return s.value, c.value


def normal(seed, purpose, traj, step, site, sub=0):
    return lib().dqo_normal(seed, purpose, traj, step, site, sub)


def hbar_reference():
    return lib().dqo_hbar_reference()


def pade_ck(p=6):
    ck = np.zeros(p + 1)
    lib().dqo_pade_ck(p, _dp(ck))
    return ck


def pade_exp(A, norm_mode=NORM_COMPLEX):
    A = np.ascontiguousarray(A, dtype=np.complex128)
    L = A.shape[0]
    E = np.zeros_like(A)
    s = lib().dqo_pade_exp(L, _dp(A.view(np.float64)), _dp(E.view(np.float64)), norm_mode)
    return E, s


def ifft(x):
    x = np.array(x, dtype=np.complex128)
    lib().dqo_ifft(len(x), _dp(x.view(np.float64)))
    return x


class System:
    """Python holder for a dqo_system (keeps the numpy buffers alive).

    rowptr/col/val is the OFF-DIAGONAL CSR; h0diag the input diagonal."""

    def __init__(self, rowptr, col, val, h0diag, m, dt, hbar=None, dot_mode=DOT_BILINEAR,
                 norm_mode=NORM_COMPLEX, noise=NOISE_NONE, ka_substeps=1, sigma=None, tau=None,
                 sigma_static=0.0, static_eps=None, seed=0, reorth=0, m_min=0, m_tol=1e-7, zz_omega=None,
                 zz_coeff=None, tk=None, corr_bra=None):
        """tk: optional Taylor-Krylov mode (p, m_B, rowptr_B, col_B, val_B, diag_B), B's off-diagonal CSR
        and diagonal."""
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self.h0diag = np.ascontiguousarray(h0diag, dtype=np.float64)
        self.n = len(self.h0diag)
        self.sigma = None if sigma is None else np.ascontiguousarray(np.broadcast_to(sigma, (self.n,)), dtype=np.float64)
        self.tau = None if tau is None else np.ascontiguousarray(np.broadcast_to(tau, (self.n,)), dtype=np.float64)
        self.static_eps = None if static_eps is None else np.ascontiguousarray(static_eps, dtype=np.float64)
        self.zz_omega = None if zz_omega is None else np.ascontiguousarray(zz_omega, dtype=np.float64)
        self.zz_coeff = None if zz_coeff is None else np.ascontiguousarray(zz_coeff, dtype=np.float64)
        self.n_osc = 0 if self.zz_omega is None else len(self.zz_omega)
        self.m = m
        self.dt = dt
        self.hbar = hbar_reference() if hbar is None else hbar
        if tk is not None:
            tp, tm, trp, tcol, tval, tdiag = tk
            self.tk = (int(tp), int(tm), np.ascontiguousarray(trp, dtype=np.int32),
                       np.ascontiguousarray(tcol, dtype=np.int32), np.ascontiguousarray(tval, dtype=np.float64),
                       np.ascontiguousarray(tdiag, dtype=np.float64))
        else:
            self.tk = (0, 0, None, None, None, None)
        self.corr_bra = None if corr_bra is None else np.ascontiguousarray(corr_bra, dtype=np.complex128)
        _ip = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))
        self.s = _System(
            self.n,
            self.rowptr.ctypes.data_as(C.POINTER(C.c_int)),
            self.col.ctypes.data_as(C.POINTER(C.c_int)),
            _dp(self.val),
            _dp(self.h0diag),
            m, dt, self.hbar, dot_mode, norm_mode, noise, ka_substeps,
            _dp(self.sigma), _dp(self.tau), float(sigma_static), _dp(self.static_eps), seed, int(reorth),
            int(m_min), float(m_tol), self.n_osc, _dp(self.zz_omega), _dp(self.zz_coeff),
            self.tk[0], self.tk[1], _ip(self.tk[2]), _ip(self.tk[3]), _dp(self.tk[4]), _dp(self.tk[5]),
            None if self.corr_bra is None else _dp(self.corr_bra.view(np.float64)),
        )

    def dense(self, diag=None):
        H = np.zeros((self.n, self.n))
        for i in range(self.n):
            for p in range(self.rowptr[i], self.rowptr[i + 1]):
                H[i, self.col[p]] += self.val[p]
        H[np.arange(self.n), np.arange(self.n)] += self.h0diag if diag is None else diag
        return H

    def traj_init(self, traj):
        eps = np.zeros(self.n)
        deps = np.zeros(self.n)
        lib().dqo_traj_init(C.byref(self.s), traj, _dp(eps), _dp(deps))
        return eps, deps

    def zz_phases(self, traj):
        """[osc][site] phase fractions of one trajectory."""
        u = np.zeros((self.n_osc, self.n), dtype=np.float32)
        for o in range(self.n_osc):
            for i in range(self.n):
                u[o, i] = lib().dqo_zz_phase(self.s.seed, traj, i, o)
        return u

    def noise_update_zz(self, step, eps, u):
        diag = np.zeros(self.n)
        u = np.ascontiguousarray(u, dtype=np.float32)
        lib().dqo_noise_update_zz(C.byref(self.s), step, _dp(np.ascontiguousarray(eps, dtype=np.float64)),
                                  u.ctypes.data_as(C.POINTER(C.c_float)), _dp(diag))
        return diag

    def noise_update(self, traj, step, eps, deps):
        diag = np.zeros(self.n)
        lib().dqo_noise_update(C.byref(self.s), traj, step, _dp(eps), _dp(deps), _dp(diag))
        return diag

    def krylov_step(self, diag, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.zeros_like(psi)
        err, nrm, s = C.c_double(), C.c_double(), C.c_int()
        rc = lib().dqo_krylov_step(C.byref(self.s), _dp(np.ascontiguousarray(diag, dtype=np.float64)),
                                   _dp(psi.view(np.float64)), _dp(out.view(np.float64)),
                                   C.byref(err), C.byref(nrm), C.byref(s))
        if rc != 0:
            raise RuntimeError(f"oracle krylov step failed ({rc})")
        return out, err.value, nrm.value, s.value

    def tk_step(self, diag, psi):
        """One Taylor-Krylov step: (psi_out, error estimate, norm before renormalisation)."""
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.zeros_like(psi)
        err, nrm = C.c_double(), C.c_double()
        rc = lib().dqo_tk_step(C.byref(self.s), _dp(np.ascontiguousarray(diag, dtype=np.float64)),
                               _dp(psi.view(np.float64)), _dp(out.view(np.float64)), C.byref(err), C.byref(nrm))
        if rc != 0:
            raise RuntimeError(f"oracle Taylor-Krylov step failed ({rc})")
        return out, err.value, nrm.value

    def krylov_step_m(self, diag, psi):
        """One step; also returns the Krylov dimension used (adaptive when m_min > 0)."""
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.zeros_like(psi)
        err, nrm, s, mu = C.c_double(), C.c_double(), C.c_int(), C.c_int()
        rc = lib().dqo_krylov_step_m(C.byref(self.s), _dp(np.ascontiguousarray(diag, dtype=np.float64)),
                                     _dp(psi.view(np.float64)), _dp(out.view(np.float64)),
                                     C.byref(err), C.byref(nrm), C.byref(s), C.byref(mu))
        if rc != 0:
            raise RuntimeError(f"oracle krylov step failed ({rc})")
        return out, err.value, mu.value

    def lanczos(self, diag, q1):
        n, m = self.n, self.m
        Q = np.zeros((m + 2, n), dtype=np.complex128)
        al = np.zeros(m + 2, dtype=np.complex128)
        be = np.zeros(m + 2, dtype=np.complex128)
        q1 = np.ascontiguousarray(q1, dtype=np.complex128)
        nav = lib().dqo_lanczos(C.byref(self.s), _dp(np.ascontiguousarray(diag, dtype=np.float64)),
                                _dp(q1.view(np.float64)), _dp(Q.view(np.float64)),
                                _dp(al.view(np.float64)), _dp(be.view(np.float64)))
        return Q, al, be, nav

    def run(self, n_traj, n_steps, psi0, pop_every=1, traj0=0, threads=0, want_final=False):
        n = self.n
        psi0 = np.ascontiguousarray(psi0, dtype=np.complex128)
        n_rec = n_steps // pop_every + 1
        pops = np.zeros((n_rec, n))
        corr = np.zeros(n_steps + 1, dtype=np.complex128)
        fin = np.zeros((n_traj, n), dtype=np.complex128) if want_final else None
        err = np.zeros(n_traj)
        ipr = np.zeros(n_steps + 1)
        rc = lib().dqo_run(C.byref(self.s), traj0, n_traj, n_steps, _dp(psi0.view(np.float64)), pop_every,
                           _dp(pops), _dp(corr.view(np.float64)),
                           _dp(fin.view(np.float64)) if fin is not None else None, _dp(err), _dp(ipr), threads)
        if rc != 0:
            raise RuntimeError(f"oracle run failed ({rc})")
        return {"pops": pops, "corr": corr, "psi_final": fin, "err": err, "ipr": ipr}


def spectrum_loss_grad(rowptr, col, val_base, cls, scales, static_eps, m, dt, psi0, n_traj, n_steps,
                       length, scale, target, want_grad=True, hbar=None, noise=NOISE_NONE, ka_substeps=1,
                       sigma=None, tau=None, seed=0, zz_omega=None, zz_coeff=None):
    """Loss sum_j (scale*Re(IDFT_length(Cbar)_j) - target_j)^2 and its gradient with respect to the
    site energies (static_eps, n) and the coupling-class scales (len(scales)).

    The off-diagonal couplings are val[p] = scales[cls[p]] * val_base[p]; Hermitian Lanczos dot,
    complex Padé norm.  Returns (loss, grad) with grad None when want_grad is False."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val_base = np.ascontiguousarray(val_base, dtype=np.float64)
    cls = np.ascontiguousarray(cls, dtype=np.int32)
    scales = np.asarray(scales, dtype=np.float64)
    val = scales[cls] * val_base if len(cls) else val_base.copy()
    eps = np.ascontiguousarray(static_eps, dtype=np.float64)
    sysm = System(rowptr, col, val, eps, m, dt, hbar=hbar, dot_mode=DOT_HERMITIAN, norm_mode=NORM_COMPLEX,
                  noise=noise, ka_substeps=ka_substeps, sigma=sigma, tau=tau, static_eps=eps, seed=seed,
                  zz_omega=zz_omega, zz_coeff=zz_coeff)
    psi0 = np.ascontiguousarray(psi0, dtype=np.complex128)
    target = np.ascontiguousarray(target, dtype=np.float64)
    assert target.shape == (length,)
    grad = np.zeros(sysm.n + len(scales)) if want_grad else None
    loss = lib().dqo_spectrum_loss_grad(C.byref(sysm.s), _dp(val_base), cls.ctypes.data_as(C.POINTER(C.c_int)),
                                        len(scales), n_traj, n_steps, _dp(psi0.view(np.float64)), length,
                                        float(scale), _dp(target), _dp(grad), 0)
    return loss, grad


def zz_coefficients(omega_invcm, J, d_omega, temperature):
    """(angular frequencies in rad/fs, amplitudes in cm^-1) of a ZZ spectral density."""
    omega_invcm = np.ascontiguousarray(omega_invcm, dtype=np.float64)
    J = np.ascontiguousarray(J, dtype=np.float64)
    w = np.zeros_like(omega_invcm)
    c = np.zeros_like(omega_invcm)
    lib().dqo_zz_coefficients(len(w), _dp(omega_invcm), _dp(J), float(d_omega), float(temperature), _dp(w), _dp(c))
    return w, c


def read_spectral_density(path):
    """A ZZ spectral-density file: first line "dOmega nOsc", then nOsc lines "omega J" (cm^-1)."""
    lines = [ln.split() for ln in open(path).read().splitlines() if ln.strip()]
    d_omega, n_osc = float(lines[0][0]), int(lines[0][1])
    rows = np.array([[float(a), float(b)] for a, b in lines[1:1 + n_osc]])
    return d_omega, rows[:, 0], rows[:, 1]
