"""The allocation-free entry point kpp_b200_rosenbrock_static (GPU).

Some callers cannot allocate device memory: a host model with a fixed device
budget, code that runs inside a stream capture that must not allocate, or a
library that is only handed its inputs and outputs.  For them the library
keeps the integrator's work arrays in a fixed device array of its own (at
most 1024 cells per call).  This test calls that entry through the C ABI
twice in a row and checks both results against the regular entry point,
kpp_b200_rosenbrock, on the same inputs, with the parity tolerance of the
other GPU tests; and checks that a batch above the maximum is refused with a
clear error.  It runs on every built mechanism: saprc99 and MCM isoprene keep
their work arrays in that device array, small_strato keeps them in registers
(the entry then needs no array at all).  The two entries run the same per-cell
arithmetic, so their results must be identical bit for bit.  The file is named
so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

from kpp_b200 import load, library_path, workloads

pytestmark = pytest.mark.gpu

_vp = ctypes.c_void_p
# Cells per call of the fixed device array: 1024, or 128 for mechanisms whose
# per-cell work arrays would make 1024 cells exceed 64 MB.
MAX_CELLS = {"small_strato": 1024, "saprc99": 1024, "mcm_isoprene": 128}
WORKLOAD = {"small_strato": "small_strato", "saprc99": "saprc99_uniform95",
            "mcm_isoprene": "mcm_isoprene"}
# Cells of the compared batch: ragged (not a multiple of a block).
NCELLS = {"small_strato": 700, "saprc99": 700, "mcm_isoprene": 100}


def _mechanisms():
    return [pytest.param(m, marks=pytest.mark.skipif(not library_path(m).exists(),
                                                     reason=f"{m} library not built"))
            for m in MAX_CELLS]


def _dev(a):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()


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
    p = lambda t: None if t is None else _vp(t.data_ptr())
    rc = f(ncells, ld, p(var), p(fix), p(temp), p(cf), p(sun), p(d0), p(d1), p(atol), p(rtol),
           ip, rp, None, p(ist), p(rst), p(ierr), _vp(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, var.cpu().numpy(), ist.cpu().numpy(), rst.cpu().numpy(), ierr.cpu().numpy()


@pytest.mark.parametrize("mech", _mechanisms())
def test_static_entry_matches_allocating_entry_twice_in_a_row(mech):
    m = load(mech)
    f = _static_entry(m)
    n = NCELLS[mech]
    wl = workloads.for_mechanism(m, WORKLOAD[mech], n, seed=31)
    t0, t1 = wl.step_bounds(0)
    var = _dev(wl.var)
    ref = m.rosenbrock(var, _dev(wl.fix), _dev(wl.temp), _dev(t0), _dev(t1), _dev(wl.atol),
                       _dev(wl.rtol), wl.ipar, wl.rpar, cfactor=_dev(wl.cfactor), sun=_dev(wl.sun))
    torch.cuda.synchronize()
    ref_var = var.cpu().numpy()
    for _ in range(2):
        rc, v, ist, rst, ierr = _call_static(m, f, wl, n)
        assert rc == 0, m.lib.kpp_b200_last_error()
        np.testing.assert_array_equal(ierr, ref.ierr.cpu().numpy())
        np.testing.assert_array_equal(v, ref_var)
        np.testing.assert_array_equal(ist, ref.istatus.cpu().numpy())
        np.testing.assert_array_equal(rst, ref.rstatus.cpu().numpy())


@pytest.mark.parametrize("mech", _mechanisms())
def test_static_entry_refuses_batches_above_its_maximum(mech):
    m = load(mech)
    f = _static_entry(m)
    cap = MAX_CELLS[mech]
    wl = workloads.for_mechanism(m, WORKLOAD[mech], cap + 1, seed=32)
    rc, *_ = _call_static(m, f, wl, cap + 1)
    assert rc == 1
    assert f"maximum of {cap} cells".encode() in m.lib.kpp_b200_last_error()
