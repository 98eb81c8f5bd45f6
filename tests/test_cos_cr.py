"""The correctly rounded cosine used by the device Update_SUN (CPU): compiled
for the host from the same source, it must equal the correctly rounded cosine
(mpmath at 200 bits, rounded to double) exactly -- an error bound of 0.5 ulp --
on 20000 seeded arguments of Update_SUN's range [-pi, pi] and its end points."""
import ctypes
import math
import shutil
import subprocess

import numpy as np
import pytest

from oracle_lib import REPO

mpmath = pytest.importorskip("mpmath")


@pytest.fixture(scope="module")
def cos_cr(tmp_path_factory):
    hdr = REPO / "kpp_b200" / "_gen" / "small_strato.cuh"
    if not hdr.exists():
        pytest.skip("generated mechanism code not present")
    out = tmp_path_factory.mktemp("cos") / "h.so"
    subprocess.run([shutil.which("g++"), "-O2", "-fPIC", "-shared", "-std=c++17", "-I",
                    str(REPO / "kpp_b200" / "csrc"), f'-DKPP_MECH_HEADER="{hdr}"',
                    str(REPO / "tests" / "host_harness.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.host_cos_cr.restype = ctypes.c_double
    lib.host_cos_cr.argtypes = [ctypes.c_double]
    return lib.host_cos_cr


def test_cosine_is_correctly_rounded_on_the_sun_range(cos_cr):
    mpmath.mp.prec = 200
    rng = np.random.default_rng(20261203)
    pi_kpp = 3.14159265358979
    xs = list(rng.uniform(-pi_kpp, pi_kpp, 20000)) + [0.0, -0.0, pi_kpp, -pi_kpp,
                                                      math.pi / 2, -math.pi / 2, math.pi / 4]
    bad = [x for x in xs if cos_cr(float(x)) != float(mpmath.cos(mpmath.mpf(float(x))))]
    assert not bad, bad[:5]
