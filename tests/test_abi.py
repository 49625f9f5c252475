"""The C-ABI library loads and exports every entry point include/dq.h
declares (no GPU needed: nothing here launches work)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"DQ_API\s+[^;(]*?\b(dq_\w+)\s*\(", txt)
    return names


@pytest.fixture(scope="module")
def lib():
    from dynaquant_b200 import build
    build.build()
    from dynaquant_b200 import _lib
    return _lib.load()


def test_header_declares_entry_points():
    names = _declared()
    assert "dq_prop_step" in names and "dq_run" in names and len(names) >= 20


def test_every_declared_symbol_is_exported(lib):
    from dynaquant_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (dq_\w+)", out))
    declared = set(_declared())
    assert declared <= exported, declared - exported
    # and nothing undeclared leaks out
    assert exported <= declared, exported - declared
    assert set(_lib.EXPORTS) == declared
    for n in declared:
        assert hasattr(lib, n)


def test_config_default_layout(lib):
    import ctypes as C
    from dynaquant_b200 import _lib
    cfg = _lib.Config()
    lib.dq_config_default(C.byref(cfg))
    assert cfg.m == 16 and cfg.n_traj == 1 and cfg.dt == 1.0 and cfg.pop_every == 1 and cfg.max_steps == 1024
    assert cfg.dot_mode == _lib.DOT_HERMITIAN and cfg.precision == _lib.PREC_MIXED and cfg.ka_substeps == 1


def test_last_error_null_context(lib):
    assert lib.dq_last_error(None) == b"null context"
    assert lib.dq_steps_done(None) == -1


def test_create_rejects_bad_config_without_gpu(lib):
    import ctypes as C
    from dynaquant_b200 import _lib
    cfg = _lib.Config()
    lib.dq_config_default(C.byref(cfg))
    h = C.c_void_p()
    cfg.n_sites = 100
    cfg.m = 40   # above the Krylov limit
    assert lib.dq_create(C.byref(cfg), C.byref(h)) == _lib.DQ_ERR_ARG
    cfg.m = 16
    cfg.reorth = 1
    cfg.dot_mode = _lib.DOT_BILINEAR   # reorthogonalisation needs the Hermitian product
    assert lib.dq_create(C.byref(cfg), C.byref(h)) == _lib.DQ_ERR_ARG
    assert h.value is None


def test_no_cpu_fallback_without_a_gpu(lib):
    # a valid configuration on a machine without a GPU is refused with a CUDA error, never run on the host
    import ctypes as C

    import pytest
    import torch

    from dynaquant_b200 import _lib
    import dynaquant_b200 as dq
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = _lib.Config()
    lib.dq_config_default(C.byref(cfg))
    cfg.n_sites = 100
    h = C.c_void_p()
    assert lib.dq_create(C.byref(cfg), C.byref(h)) == _lib.DQ_ERR_CUDA
    assert h.value is None
    with pytest.raises(dq.DQError):
        dq.Propagator(100, m=8, n_traj=2)
