"""Constants of the step against the reference's own functions, compiled from its
cppUtility.cpp into oracle/_ref (skipped where the reference's sources are absent):
hbar and the exponent coefficient (get_neg_inv_hbar_imag, propagate.cu:92-93) and the
Taylor-Krylov coefficients tau^k / k! (powComplex / helperFactorial,
taylorKrylovClass.cu:202-206), against the oracle's and the library's formulas."""
import ctypes as C
import math
import os

import pytest

pytestmark = pytest.mark.skipif(not os.path.exists("/root/reference/cppUtility.cpp"),
                                reason="reference sources absent")


def _ref():
    from oracle import oracle as O
    O.build()
    L = C.CDLL(O.REF_INFILE)
    L.ref_exp_coeff.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.ref_taylor_coeff.argtypes = [C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return O, L


def _coeff(L, fn, *args):
    re, im = C.c_double(), C.c_double()
    fn(*args, C.byref(re), C.byref(im))
    return complex(re.value, im.value)


def test_hbar_is_the_references_own():
    O, L = _ref()
    import dynaquant_b200 as dq
    e1 = _coeff(L, L.ref_exp_coeff, 1.0)
    assert e1.real == 0.0
    # the reference stores -1/hbar; hbar itself is bit-identical in the oracle and the library
    assert -1.0 / e1.imag == pytest.approx(O.hbar_reference(), rel=2e-16)
    assert O.hbar_reference() == dq.reference_hbar()


@pytest.mark.parametrize("dt", [0.5, 1.0, 2.0])
def test_exponent_and_taylor_coefficients_match_the_reference(dt):
    O, L = _ref()
    hbar = O.hbar_reference()
    tau = complex(0.0, -dt / hbar)   # the oracle's and the library's tau = -i dt / hbar
    assert _coeff(L, L.ref_exp_coeff, dt) == pytest.approx(tau, rel=4e-16)
    pw, fact = complex(1.0, 0.0), 1.0
    for k in range(12):
        if k:
            pw, fact = pw * tau, fact * k
        ref = _coeff(L, L.ref_taylor_coeff, dt, k)
        mine = complex(pw.real / fact, pw.imag / fact)
        assert abs(mine - ref) <= 1e-15 * abs(ref) * (k + 1), (k, mine, ref)
    assert math.isfinite(abs(ref))
