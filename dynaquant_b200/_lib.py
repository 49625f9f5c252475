"""ctypes binding of libdq.so (include/dq.h).

The library is built in-tree (dynaquant_b200/build.py).  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdq.so")

DQ_OK, DQ_ERR_ARG, DQ_ERR_CUDA, DQ_ERR_BREAKDOWN, DQ_ERR_NAN, DQ_ERR_TIMEOUT, DQ_ERR_SCALING, DQ_ERR_STATE, \
    DQ_ERR_SINGULAR = range(9)
NOISE_NONE, NOISE_GAUSS, NOISE_OU, NOISE_ZZ = 0, 1, 2, 3
DOT_BILINEAR, DOT_HERMITIAN = 0, 1
NORM_REAL_ONLY, NORM_COMPLEX = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
KIND_NAMES = ["noise", "spmm_alpha", "axpy_beta", "spmm_norm", "pade", "combine", "pop", "fused_iter"]

# every symbol include/dq.h declares
EXPORTS = [
    "dq_config_default", "dq_create", "dq_destroy", "dq_last_error", "dq_get_stream",
    "dq_set_hamiltonian_csr", "dq_set_coupling_classes", "dq_set_noise_params", "dq_set_static_energies",
    "dq_set_zz_spectral_density", "dq_set_taylor_krylov", "dq_set_ipr", "dq_get_ipr", "dq_write_ipr",
    "dq_set_correlation_bra", "dq_set_trajectory_offset", "dq_get_observable_sums", "dq_set_observable_sums",
    "dq_set_initial_state", "dq_set_initial_dipole", "dq_reset", "dq_prop_step", "dq_run_plain", "dq_run", "dq_get_populations",
    "dq_get_correlation", "dq_get_states", "dq_get_error_accum", "dq_steps_done", "dq_get_spectrum",
    "dq_get_noise_state", "dq_set_line_dressing", "dq_profile_step", "dq_set_tiling", "dq_get_tiling", "dq_autotune", "dq_time_iteration", "dq_time_gather_floor",
    "dq_debug_set_wait_cycles", "dq_krylov_step_static", "dq_adjoint_setup", "dq_forward", "dq_backward", "dq_forward_shard", "dq_forward_reduced",
    "dq_group_create", "dq_group_destroy", "dq_group_last_error", "dq_group_run", "dq_group_run_timed",
    "dq_write_populations", "dq_write_states", "dq_write_spectrum", "dq_write_spectrum_mean",
    # include/dq_host.h
    "dq_infile_defaults", "dq_infile_parse", "dq_infile_split_line", "dq_infile_run",
]

HOST_PATH_MAX = 1024
ENS_AVG_NONE, ENS_AVG_FIRST, ENS_AVG_CONTINUATION = 0, 1, 2
SIM_CONST_HAM, SIM_HSR, SIM_KUBO_ANDERSON, SIM_ZZ_REAL_NOISE, SIM_ZZ_COMPLEX_NOISE = range(5)
PROP_LANCZOS, PROP_TAYLOR_LANCZOS = 0, 1


class InFile(C.Structure):
    """struct dq_infile (include/dq_host.h)."""
    _fields_ = [
        ("dt", C.c_double), ("totalsteps", C.c_int), ("ensembleavgmode", C.c_int), ("ensembleruns", C.c_int),
        ("m", C.c_int), ("ka_substeps", C.c_int), ("absorbspec", C.c_int), ("cdspec", C.c_int),
        ("lineshapedress", C.c_int), ("gausswidth", C.c_double), ("dostatelooping", C.c_int),
        ("stepsperloop", C.c_int), ("writeoutpops", C.c_int), ("printallpops", C.c_int),
        ("writebinarypops", C.c_int), ("printpop", C.c_int * 10), ("print_partic", C.c_int),
        ("writeoutstates", C.c_int), ("initstate", C.c_int), ("initfromfile", C.c_int), ("propmode", C.c_int),
        ("simtype", C.c_int), ("staticdis", C.c_int), ("sigmastatdis", C.c_double), ("temperature", C.c_double),
        ("debug_diags", C.c_int), ("tk_p", C.c_int), ("tk_m_aux", C.c_int),
    ] + [(nm, C.c_char * HOST_PATH_MAX) for nm in (
        "hamfile", "statefile", "outfile", "tkmatfile", "outfolder", "hsr_stddevfile", "ka_paramsfile",
        "zz_specd_file", "dipolefile", "posfile", "initstatefile")] + [
        ("precision", C.c_int), ("seed", C.c_uint64), ("pop_every", C.c_int),
        ("n_assignments", C.c_int), ("n_unknown", C.c_int),
    ]


class Config(C.Structure):
    _fields_ = [
        ("n_sites", C.c_int),
        ("m", C.c_int),
        ("n_traj", C.c_int),
        ("dt", C.c_double),
        ("hbar", C.c_double),
        ("noise_model", C.c_int),
        ("ka_substeps", C.c_int),
        ("sigma_static", C.c_double),
        ("seed", C.c_uint64),
        ("dot_mode", C.c_int),
        ("norm_mode", C.c_int),
        ("precision", C.c_int),
        ("reorth", C.c_int),
        ("pop_every", C.c_int),
        ("m_min", C.c_int),
        ("m_tol", C.c_double),
        ("max_steps", C.c_int),
        ("device", C.c_int),
    ]


class CDouble(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


_lib = None


def load(path: str = LIB_PATH):
    """Loads libdq.so and declares its signatures; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m dynaquant_b200.build` "
                           "(the propagator has no CPU fallback)")
    L = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    cfgp = C.POINTER(Config)
    L.dq_config_default.argtypes = [cfgp]
    L.dq_config_default.restype = None
    L.dq_create.argtypes = [cfgp, C.POINTER(vp)]
    L.dq_destroy.argtypes = [vp]
    L.dq_destroy.restype = None
    L.dq_last_error.argtypes = [vp]
    L.dq_last_error.restype = C.c_char_p
    L.dq_get_stream.argtypes = [vp]
    L.dq_get_stream.restype = vp
    L.dq_set_hamiltonian_csr.argtypes = [vp, C.c_int, ip, ip, dp]
    L.dq_set_coupling_classes.argtypes = [vp, ip, C.c_int, dp]
    L.dq_set_noise_params.argtypes = [vp, dp, dp]
    L.dq_set_zz_spectral_density.argtypes = [vp, C.c_int, dp, dp, C.c_double, C.c_double]
    L.dq_set_taylor_krylov.argtypes = [vp, C.c_int, C.c_int, ip, ip, dp]
    L.dq_set_ipr.argtypes = [vp, C.c_int]
    L.dq_set_trajectory_offset.argtypes = [vp, C.c_int]
    L.dq_set_correlation_bra.argtypes = [vp, dp]
    L.dq_get_observable_sums.argtypes = [vp, dp, dp, dp]
    L.dq_set_observable_sums.argtypes = [vp, dp, dp, dp, C.c_int]
    L.dq_get_ipr.argtypes = [vp, dp, C.POINTER(C.c_int)]
    L.dq_write_ipr.argtypes = [vp, C.c_char_p]
    L.dq_set_static_energies.argtypes = [vp, dp]
    L.dq_set_initial_state.argtypes = [vp, dp]
    L.dq_set_initial_dipole.argtypes = [vp, dp]
    L.dq_reset.argtypes = [vp]
    L.dq_prop_step.argtypes = [vp, C.c_int, C.c_int, vp, vp, dp]
    L.dq_run_plain.argtypes = [vp, C.c_int]
    L.dq_run.argtypes = [vp, C.c_int]
    L.dq_get_populations.argtypes = [vp, dp, ip]
    L.dq_get_correlation.argtypes = [vp, dp, ip]
    L.dq_get_states.argtypes = [vp, dp]
    L.dq_get_error_accum.argtypes = [vp, dp]
    L.dq_steps_done.argtypes = [vp]
    L.dq_steps_done.restype = C.c_int
    L.dq_get_spectrum.argtypes = [vp, C.c_int, dp]
    L.dq_set_line_dressing.argtypes = [vp, C.c_double]
    L.dq_get_noise_state.argtypes = [vp, C.c_int, dp, dp]
    L.dq_profile_step.argtypes = [vp, C.c_int, dp, ip, C.c_int]
    L.dq_set_tiling.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L.dq_get_tiling.argtypes = [vp, ip, ip, ip, ip, ip, ip]
    L.dq_autotune.argtypes = [vp, C.c_int, dp]
    L.dq_time_iteration.argtypes = [vp, C.c_int, dp]
    L.dq_time_gather_floor.argtypes = [vp, C.c_int, dp]
    L.dq_debug_set_wait_cycles.argtypes = [vp, C.c_int]
    L.dq_krylov_step_static.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, C.c_int, C.c_double, C.c_double, C.c_int,
                                        C.c_int, vp, dp, C.c_char_p, C.c_int]
    L.dq_adjoint_setup.argtypes = [vp, C.c_int, C.c_int, C.c_double, dp, C.c_int]
    L.dq_forward.argtypes = [vp, dp]
    L.dq_backward.argtypes = [vp, dp, dp]
    L.dq_forward_shard.argtypes = [vp, dp]
    L.dq_forward_reduced.argtypes = [vp, dp, C.c_int, C.POINTER(C.c_double)]
    L.dq_group_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
    L.dq_group_destroy.argtypes = [vp]
    L.dq_group_destroy.restype = None
    L.dq_group_last_error.argtypes = [vp]
    L.dq_group_last_error.restype = C.c_char_p
    L.dq_group_run.argtypes = [vp, C.c_int]
    L.dq_group_run_timed.argtypes = [vp, C.c_int, dp]
    L.dq_write_populations.argtypes = [vp, C.c_char_p, C.c_int, C.c_int]
    L.dq_write_states.argtypes = [vp, C.c_char_p]
    L.dq_write_spectrum.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_double]
    L.dq_write_spectrum_mean.argtypes = [C.POINTER(vp), C.c_int, dp, C.c_char_p, C.c_char_p]
    inp = C.POINTER(InFile)
    L.dq_infile_defaults.argtypes = [inp]
    L.dq_infile_defaults.restype = None
    L.dq_infile_parse.argtypes = [C.c_char_p, inp, C.c_char_p, C.c_int]
    L.dq_infile_run.argtypes = [inp, C.c_char_p, C.c_int, C.c_char_p, C.c_int]
    L.dq_infile_split_line.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_int]
    for name in EXPORTS:
        if name not in ("dq_config_default", "dq_destroy", "dq_last_error", "dq_get_stream", "dq_steps_done",
                        "dq_group_destroy", "dq_group_last_error", "dq_infile_defaults"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def dptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


class DQError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dq error {code}: {msg}")
        self.code = code
