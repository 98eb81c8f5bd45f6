"""The controllers' pow on the GPU (kpp_pow_cr, kpp_b200/csrc/kpp_ratelaws.cuh).

The device evaluation must equal the host build of the same source bit for
bit (the host build is tested correctly rounded against mpmath in
tests/test_pow_cr.py), on the same argument kinds, and so be correctly
rounded on the device.  How often the CUDA math library's pow differs from the
correctly rounded value on the same arguments is reported, not asserted: it
is why the controllers do not call it.
"""
import ctypes
import shutil
import subprocess

import numpy as np
import pytest
import torch

from kpp_b200.build import LIB
from oracle_lib import REPO
from test_pow_cr import controller_cases, wide_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def host_pow(tmp_path_factory):
    hdr = REPO / "kpp_b200" / "_gen" / "small_strato.cuh"
    out = tmp_path_factory.mktemp("pow") / "h.so"
    subprocess.run([shutil.which("g++"), "-O2", "-fPIC", "-shared", "-std=c++17", "-I",
                    str(REPO / "kpp_b200" / "csrc"), f'-DKPP_MECH_HEADER="{hdr}"',
                    str(REPO / "tests" / "host_harness.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.host_pow_cr.restype = ctypes.c_double
    lib.host_pow_cr.argtypes = [ctypes.c_double, ctypes.c_double]
    return lib.host_pow_cr


def device_pow(x, y, which):
    lib = ctypes.CDLL(str(LIB / "libkpp_b200_util.so"))
    f = lib.kpp_b200_pow_batch
    f.argtypes = [ctypes.c_longlong] + [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_void_p]
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    yd = torch.tensor(y, dtype=torch.float64, device="cuda")
    out = torch.empty_like(xd)
    assert f(len(x), xd.data_ptr(), yd.data_ptr(), out.data_ptr(), which,
             torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("kind", ["controller", "wide"])
def test_device_pow_equals_host_build(host_pow, kind):
    rng = np.random.default_rng(20261204 if kind == "controller" else 20261205)
    xs, ys = controller_cases(rng, 1000) if kind == "controller" else wide_cases(rng, 3000)
    xs = [float(v) for v in xs] + [-2.0, -1.5, -0.7, 9.0, 2.0, 0.0, 1.0]
    ys = [float(v) for v in ys] + [3.0, 5.0, 4.0, 0.5, -10.0, 2.0, 7.5]
    dev = device_pow(xs, ys, 0)
    host = np.array([host_pow(x, y) for x, y in zip(xs, ys)])
    np.testing.assert_array_equal(dev.view(np.int64), host.view(np.int64))
    cuda = device_pow(xs, ys, 1)
    print(f"\n{kind}: {len(xs)} arguments; CUDA's pow differs from the correctly rounded "
          f"value on {int((cuda != host).sum())}")
