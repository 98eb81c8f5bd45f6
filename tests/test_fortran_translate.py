"""kpp_b200/gen/fortran.py: Fortran 90 rate expressions to C with Fortran's
literal kinds and precedence.  Translated expressions are compiled with gcc
and evaluated against numpy evaluations written out with the same kinds
(float32 for default-real literals, float64 for D literals and REAL(dp)
variables)."""
import ctypes
import ctypes.util
import subprocess

import numpy as np
import pytest

from kpp_b200.gen.fortran import F32, F64, INT, Context, FortranError, translate_expr

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.log10f.restype = ctypes.c_float
_libm.log10f.argtypes = [ctypes.c_float]
T = 287.3
M = 2.1e19
f32 = np.float32

CASES = [
    # (Fortran, numpy value with Fortran kinds)
    ("2.7E-12*EXP(360./TEMP)", float(f32(2.7e-12)) * np.exp(360.0 / T)),
    ("1.7D-12*EXP(-940/TEMP)", 1.7e-12 * np.exp(-940 / T)),
    ("5.6E-34*M*(TEMP/300.)**(-2.6)", float(f32(5.6e-34)) * M * (T / 300.0) ** float(f32(-2.6))),
    ("-2.0**2", -4.0),                                         # -(2**2)
    ("(TEMP/300.)**2", (T / 300.0) * (T / 300.0)),            # integer power: a product
    ("10.**(LOG10(0.35)/(1.+(LOG10(TEMP)/0.75)**(2.)))",
     10.0 ** (float(f32(_libm.log10f(0.35)))     # LOG10 of a default real: log10f
              / (1.0 + (np.log10(T) / float(f32(0.75))) ** 2.0))),
    ("0.21*0.5", float(f32(0.21) * f32(0.5))),               # single-precision product
    ("1/2 + 3/2", 1.0),                                        # integer division
    ("KRO2NO*0.917", 1.5e-11 * float(f32(0.917))),
]


def c_eval(exprs):
    ctx = Context(variables={"TEMP": ("TEMP", F64), "M": ("M", F64), "KRO2NO": ("KRO2NO", F64)})
    body = "".join(f'  printf("%.17g\\n", (double)({translate_expr(e, ctx).text}));\n'
                   for e in exprs)
    src = ("#include <math.h>\n#include <stdio.h>\nint main(void) {\n"
           f"  double TEMP = {T!r}, M = {M!r}, KRO2NO = 1.5e-11;\n{body}  return 0;\n}}\n")
    out = subprocess.run(["gcc", "-O", "-x", "c", "-", "-lm", "-o", "/tmp/kpp_f90_eval"],
                         input=src, text=True, capture_output=True)
    assert out.returncode == 0, out.stderr
    res = subprocess.run(["/tmp/kpp_f90_eval"], capture_output=True, text=True, check=True)
    return [float(x) for x in res.stdout.split()]


def test_values_follow_fortran_kinds():
    got = c_eval([c for c, _ in CASES])
    for (src, want), g in zip(CASES, got):
        assert g == pytest.approx(want, rel=2e-15), src


def test_kinds_and_errors():
    ctx = Context()
    assert translate_expr("3", ctx).kind == INT
    assert translate_expr("3.", ctx).kind == F32
    assert translate_expr("3.D0", ctx).kind == F64
    assert translate_expr("EXP(2.5)", ctx).text == "expf(2.5f)"
    with pytest.raises(FortranError):
        translate_expr("EXP(2)", ctx)
    with pytest.raises(FortranError):
        translate_expr("1.0 +", ctx)
