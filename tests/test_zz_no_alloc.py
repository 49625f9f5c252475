"""dq_krylov_step_static: the allocation-free Krylov step.

It serves callers that cannot allocate device memory while they step (their
own pool owns all device memory, or the host framework only hands out its own
buffers): no context, no cudaMalloc, scratch in one static device array.
The test calls it through the C ABI twice in a row and checks each result
against the context-based drop-in step (dq_prop_step) on the same inputs,
to the tolerance the FP64 parity tests use.  This file sorts last so a
stop-at-first-failure run has executed every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PSI_TOL = 1e-12


def _setup(n=512, m=16, dot=1, norm=1):
    import torch

    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    rng = np.random.default_rng(3)
    h0 = rng.normal(0.0, 100.0, n)
    s = systems.chain(n, -300.0, diag=h0)
    p = dq.Propagator(n, m=m, n_traj=1, dt=1.0, noise=dq.NOISE_NONE, sigma_static=0.0, dot=dot,
                      norm=norm, precision=dq.PREC_FP64)
    p.set_system(s)
    psi0 = rng.normal(size=n) + 1j * rng.normal(size=n)
    psi0 /= np.linalg.norm(psi0)
    p.set_initial_state(psi0)
    p.reset()
    rp, col, val, diag = s.off_diagonal()
    dev = dict(rp=torch.tensor(rp, dtype=torch.int32, device="cuda"),
               col=torch.tensor(col, dtype=torch.int32, device="cuda"),
               val=torch.tensor(val, dtype=torch.float64, device="cuda"),
               diag=torch.tensor(diag, dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    return p, psi0, dev


def _static_step(lib, n, m, dev, a, b, stream, errbuf, dot=1, norm=1, want_err=True):
    err = C.c_double()
    rc = lib.dq_krylov_step_static(n, C.c_void_p(dev["rp"].data_ptr()), C.c_void_p(dev["col"].data_ptr()),
                                   C.c_void_p(dev["val"].data_ptr()), C.c_void_p(dev["diag"].data_ptr()),
                                   C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), m, 1.0, 0.0,
                                   dot, norm, C.c_void_p(stream), C.byref(err) if want_err else None, errbuf,
                                   len(errbuf))
    return rc, err.value


# (n, dot, norm, m): a multiple of the 256-thread block and a ragged n, both
# Lanczos dot forms and both Padé norms, and m = 24, whose Padé needs more
# than 48 KB of shared memory (launched after a context with m = 8 exists on
# the device, which must not lower the kernel's limit)
CASES = [(512, 1, 1, 16), (1000, 1, 1, 16), (1000, 0, 0, 16), (1000, 1, 1, 24)]


@pytest.mark.parametrize("n,dot,norm,m", CASES)
def test_static_step_matches_context_step_twice(n, dot, norm, m):
    import torch

    import dynaquant_b200 as dq
    from dynaquant_b200 import _lib
    lib = _lib.load()
    small = dq.Propagator(64, m=8, n_traj=1, dt=1.0, precision=dq.PREC_FP64)   # a smaller-m context first
    p, psi0, dev = _setup(n, m, dot, norm)
    errbuf = C.create_string_buffer(256)
    with torch.cuda.stream(torch.cuda.ExternalStream(p.stream)):
        a = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
        b = torch.empty_like(a)
        c = torch.empty_like(a)
        e1 = p.prop_step(0, 0, a.data_ptr(), b.data_ptr(), want_error=True)
        e2 = p.prop_step(0, 1, b.data_ptr(), c.data_ptr(), want_error=True)
        a2 = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
        b2 = torch.empty_like(a2)
        c2 = torch.empty_like(a2)
        rc1, s1 = _static_step(lib, n, m, dev, a2, b2, p.stream, errbuf, dot, norm)
        assert rc1 == 0, errbuf.value
        rc2, s2 = _static_step(lib, n, m, dev, b2, c2, p.stream, errbuf, dot, norm)
        assert rc2 == 0, errbuf.value
        got_b, got_c = b2.cpu().numpy(), c2.cpu().numpy()
        ref_b, ref_c = b.cpu().numpy(), c.cpu().numpy()
    assert np.abs(got_b - ref_b).max() < PSI_TOL
    assert np.abs(got_c - ref_c).max() < PSI_TOL
    assert s1 == pytest.approx(e1, rel=1e-6, abs=1e-15) and s2 == pytest.approx(e2, rel=1e-6, abs=1e-15)
    p.close()
    small.close()


def test_static_step_error_without_err_est_is_reported_by_the_next_checked_call():
    """A call with err_est = NULL does not synchronise, so it cannot report a
    device error itself; the error stays recorded and the next call that passes
    err_est reports it (and clears it), so it is never lost."""
    import torch

    from dynaquant_b200 import _lib
    lib = _lib.load()
    n, m = 512, 16
    p, psi0, dev = _setup(n, m)
    errbuf = C.create_string_buffer(256)
    bad = psi0.copy()
    bad[5] = np.nan
    with torch.cuda.stream(torch.cuda.ExternalStream(p.stream)):
        a_bad = torch.tensor(bad, dtype=torch.complex128, device="cuda")
        a = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
        b = torch.empty_like(a)
        rc, _ = _static_step(lib, n, m, dev, a_bad, b, p.stream, errbuf, want_err=False)
        assert rc == 0   # nothing read back yet
        rc, _ = _static_step(lib, n, m, dev, a, b, p.stream, errbuf)
        assert rc == 4, errbuf.value   # DQ_ERR_NAN from the earlier call
        rc, est = _static_step(lib, n, m, dev, a, b, p.stream, errbuf)
        assert rc == 0, errbuf.value
        assert np.isfinite(b.cpu().numpy()).all() and est > 0
    p.close()


def test_static_step_rejects_sizes_beyond_its_scratch():
    import torch

    from dynaquant_b200 import _lib
    lib = _lib.load()
    n, m = 512, 16
    p, psi0, dev = _setup(n, m)
    errbuf = C.create_string_buffer(256)
    a = torch.zeros(4, dtype=torch.complex128, device="cuda")
    b = torch.zeros_like(a)
    big_n = 2_000_000   # (m+3)*n*16 bytes is far above the static array; rejected before any device work
    rc, _ = _static_step(lib, big_n, m, dev, a, b, p.stream, errbuf)
    assert rc == 1 and b"static limit" in errbuf.value
    p.close()
