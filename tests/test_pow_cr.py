"""The correctly rounded pow of the integrators' controllers (CPU):
kpp_pow_cr (kpp_b200/csrc/kpp_ratelaws.cuh), compiled for the host from the
same source, must equal x^y correctly rounded (mpmath at 200 bits, rounded to
double) exactly -- an error bound of 0.5 ulp -- on seeded arguments of every
kind the controllers pass (error norms to the powers -1/ELO and -1/4 of
int/rosenbrock.c, int/sdirk.c and int/runge_kutta.c, Newton contraction
rates to small integer powers and to -1/(k+1)), rate-law-like powers
(T/300)^C, and a wide sweep of magnitudes; negative bases with integer
exponents; and return the C library's values on the special arguments.

The C library's own pow, which the reference calls, is not correctly rounded
everywhere: the count of its differences is reported, not asserted.
"""
import ctypes
import math
import shutil
import subprocess

import numpy as np
import pytest

from oracle_lib import REPO

mpmath = pytest.importorskip("mpmath")


@pytest.fixture(scope="module")
def pow_cr(tmp_path_factory):
    hdr = REPO / "kpp_b200" / "_gen" / "small_strato.cuh"
    if not hdr.exists():
        pytest.skip("generated mechanism code not present")
    out = tmp_path_factory.mktemp("pow") / "h.so"
    subprocess.run([shutil.which("g++"), "-O2", "-fPIC", "-shared", "-std=c++17", "-I",
                    str(REPO / "kpp_b200" / "csrc"), f'-DKPP_MECH_HEADER="{hdr}"',
                    str(REPO / "tests" / "host_harness.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.host_pow_cr.restype = ctypes.c_double
    lib.host_pow_cr.argtypes = [ctypes.c_double, ctypes.c_double]
    return lib.host_pow_cr


def _libm_pow():
    libm = ctypes.CDLL("libm.so.6")
    libm.pow.restype = ctypes.c_double
    libm.pow.argtypes = [ctypes.c_double, ctypes.c_double]
    return libm.pow


def _cr(x: float, y: float) -> float:
    mpmath.mp.prec = 200
    v = mpmath.power(mpmath.mpf(abs(x)), mpmath.mpf(y))
    if x < 0 and float(y) % 2.0 == 1.0:
        v = -v
    return float(v)


def controller_cases(rng, n):
    xs, ys = [], []
    for y in (-1 / 3, -1 / 4, -1 / 5, -1 / 6, -1 / 2, -0.25, 1 / 3, 1 / 4, 1 / 5):
        xs += list(10 ** rng.uniform(-8, 8, n))
        ys += [y] * n
    for k in range(1, 9):  # theta^(Nit - it), qn^(-1/(1 + Nit - it))
        xs += list(rng.uniform(0.0, 1.0, n // 4))
        ys += [float(k)] * (n // 4)
        xs += list(10 ** rng.uniform(-6, 2, n // 4))
        ys += [-1.0 / (1 + k)] * (n // 4)
    return xs, ys


def wide_cases(rng, n):
    x = 10 ** rng.uniform(-300, 300, n)
    y = rng.uniform(-1.0, 1.0, n) * 700.0 / np.abs(np.log(x))
    t = rng.uniform(180.0, 330.0, n) / 300.0
    c = np.round(rng.uniform(-10.0, 10.0, n), 2)
    near1 = 1.0 + rng.uniform(-1e-6, 1e-6, n)
    yy = rng.uniform(-50.0, 50.0, n)
    return (list(x) + list(t) + list(near1), list(y) + list(c) + list(yy))


@pytest.mark.parametrize("kind", ["controller", "wide"])
def test_pow_is_correctly_rounded(pow_cr, kind):
    rng = np.random.default_rng(20261204 if kind == "controller" else 20261205)
    xs, ys = controller_cases(rng, 1000) if kind == "controller" else wide_cases(rng, 3000)
    libm_pow = _libm_pow()
    bad, libm_off = [], 0
    for x, y in zip(xs, ys):
        x, y = float(x), float(y)
        ref = _cr(x, y)
        if pow_cr(x, y) != ref:
            bad.append((x, y))
        libm_off += libm_pow(x, y) != ref
    print(f"\n{kind}: {len(xs)} arguments; the C library's pow differs from the correctly "
          f"rounded value on {libm_off}")
    assert not bad, bad[:5]


def test_exact_and_negative_bases(pow_cr):
    cases = [(2.0, 10.0), (2.0, -10.0), (9.0, 0.5), (1e-300, 0.5), (3.0, 2.0), (10.0, -1.0),
             (0.1, 3.0), (7.0, 1.0), (-2.0, 3.0), (-2.0, 2.0), (-3.0, -1.0), (-1.5, 5.0),
             (-0.7, 4.0), (-1.0, 1e17), (-1.0, 3.0), (1.0 + 2 ** -52, 2.0 ** 52),
             (float(2 ** 26 + 1), 2.0), (float(2 ** 27 - 1), 2.0)]
    for x, y in cases:
        assert pow_cr(x, y) == _cr(x, y), (x, y)


def test_special_arguments_follow_the_c_library(pow_cr):
    libm_pow = _libm_pow()
    inf, nan = math.inf, math.nan
    for x, y in [(0.0, 2.0), (0.0, -2.0), (-0.0, 3.0), (-0.0, -3.0), (0.0, 0.0), (inf, 2.0),
                 (inf, -2.0), (-inf, 3.0), (2.0, inf), (0.5, inf), (2.0, -inf), (1.0, nan),
                 (nan, 0.0), (nan, 2.0), (2.0, nan), (-2.0, 0.5), (-8.0, 1 / 3), (1e300, 3.0),
                 (1e-300, 3.0), (10.0, 400.0)]:
        a, b = pow_cr(x, y), libm_pow(x, y)
        assert (math.isnan(a) and math.isnan(b)) or (a == b and math.copysign(1, a) ==
                                                       math.copysign(1, b)), (x, y, a, b)
