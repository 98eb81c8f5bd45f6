"""The allocation-free entry point kpp_b200_rosenbrock_static (GPU).

Some callers cannot allocate device memory: a host model with a fixed device
budget, code that runs inside a stream capture that must not allocate, or a
library that is only handed its inputs and outputs.  For them the library
keeps the integrator's work arrays in a fixed device array of its own (at
most 1024 cells per call).  This test calls that entry through the C ABI
twice in a row and checks both results against the regular entry point,
kpp_b200_rosenbrock, on the same inputs, with the parity tolerance of the
other GPU tests; and checks that a batch above the maximum is refused with a
clear error.  It runs on saprc99, whose kernel keeps its work arrays in
scratch memory.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

from kpp_b200 import load, workloads
from parity import REL_TOL, max_rel_err

pytestmark = pytest.mark.gpu

_vp = ctypes.c_void_p
MAX_CELLS = 1024


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _static_entry(m):
    f = m.lib.kpp_b200_rosenbrock_static
    f.argtypes = ([ctypes.c_int, ctypes.c_int] + [_vp] * 9
                  + [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)] + [_vp] * 5)
    f.restype = ctypes.c_int
    return f


def _call_static(m, f, wl, ncells):
    t0, t1 = wl.step_bounds(0)
    var = _dev(wl.var)
    ld = var.shape[1]
    ist = torch.empty(8, ld, dtype=torch.int32, device="cuda")
    rst = torch.empty(2, ld, dtype=torch.float64, device="cuda")
    ierr = torch.empty(ld, dtype=torch.int32, device="cuda")
    keep = [_dev(x) for x in (wl.fix, wl.temp, wl.cfactor, wl.sun, t0, t1, wl.atol, wl.rtol)]
    fix, temp, cf, sun, d0, d1, atol, rtol = keep
    ip = (ctypes.c_int * 20)(*wl.ipar)
    rp = (ctypes.c_double * 20)(*wl.rpar)
    p = lambda t: _vp(t.data_ptr())
    rc = f(ncells, ld, p(var), p(fix), p(temp), p(cf), p(sun), p(d0), p(d1), p(atol), p(rtol),
           ip, rp, None, p(ist), p(rst), p(ierr), _vp(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, var.cpu().numpy(), ist.cpu().numpy(), rst.cpu().numpy(), ierr.cpu().numpy()


def test_static_entry_matches_allocating_entry_twice_in_a_row():
    m = load("saprc99")
    f = _static_entry(m)
    wl = workloads.for_mechanism(m, "saprc99_uniform95", 700, seed=31)
    t0, t1 = wl.step_bounds(0)
    var = _dev(wl.var)
    ref = m.rosenbrock(var, _dev(wl.fix), _dev(wl.temp), _dev(t0), _dev(t1), _dev(wl.atol),
                       _dev(wl.rtol), wl.ipar, wl.rpar, cfactor=_dev(wl.cfactor), sun=_dev(wl.sun))
    torch.cuda.synchronize()
    ref_var = var.cpu().numpy()
    for _ in range(2):
        rc, v, ist, rst, ierr = _call_static(m, f, wl, 700)
        assert rc == 0, m.lib.kpp_b200_last_error()
        np.testing.assert_array_equal(ierr, ref.ierr.cpu().numpy())
        assert max_rel_err(v, ref_var) <= REL_TOL
        np.testing.assert_array_equal(ist, ref.istatus.cpu().numpy())
        assert max_rel_err(rst, ref.rstatus.cpu().numpy(), floor=0.0) <= REL_TOL


def test_static_entry_refuses_batches_above_its_maximum():
    m = load("saprc99")
    f = _static_entry(m)
    wl = workloads.for_mechanism(m, "saprc99_uniform95", MAX_CELLS + 1, seed=32)
    rc, *_ = _call_static(m, f, wl, MAX_CELLS + 1)
    assert rc == 1
    assert b"maximum of 1024 cells" in m.lib.kpp_b200_last_error()
