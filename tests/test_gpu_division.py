"""The division through a reciprocal of the warp-per-cell kernel's backward
substitution (kpp_b200/csrc/kpp_div.cuh) against the division itself (GPU).

Markstein's correction step with a correctly rounded reciprocal gives the
correctly rounded quotient while its operands stay in a guarded range, and the
guard hands every other operand pair to the division; so the result must equal
a / b in every bit, for random operands of every magnitude, divisors with
significands near all ones or near a power of two, and quotients next to
representable numbers (the cases where rounding is hardest).
"""
import ctypes

import pytest

from kpp_b200.build import LIB

pytestmark = pytest.mark.gpu

CASES = [(-300, 300, 0), (-1022, 1023, 0), (-300, 300, 1), (-300, 300, 2), (-300, 300, 3),
         (-1022, 1023, 1), (-1022, 1023, 3)]


@pytest.mark.parametrize("emin,emax,mode", CASES)
def test_reciprocal_division_equals_division(emin, emax, mode):
    lib = ctypes.CDLL(str(LIB / "libkpp_b200_util.so"))
    f = lib.kpp_b200_check_division
    f.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    f.restype = ctypes.c_longlong
    n = 1 << 30
    assert f(20261204 + mode, n, emin, emax, mode) == 0
