"""The SDIRK integrator of kpp_b200 (kpp_sdirk.cuh), compiled for the host,
against the reference's own C SDIRK (int/sdirk.c) on the same mechanism:
bit for bit, for every method, the control cases and error paths, in one
process (so that no state carried between calls, such as stage vectors a
failed step did not write, goes unnoticed).

Both sides run on the CPU with the same compiler and libm, so any difference
is an error of the restatement.  The GPU tests (test_gpu_sdirk.py) then only
have CUDA's last-ulp libm differences to account for.
"""
import ctypes
import shutil
import subprocess

import numpy as np
import pytest

from kpp_b200 import workloads
from oracle_lib import REPO, OracleLib, SdirkOracle, _p, ensure_built, sdirk_lib_path

MECHS = {"small_strato": 64, "saprc99": 16, "mcm_isoprene": 4}


def _controls(method=3, scalar_tol=True, **kw):
    ic, rc = [0] * 20, [0.0] * 20
    ic[1] = 1 if scalar_tol else 0
    ic[2] = method
    slots = {"max_steps": (ic, 3), "newton_maxit": (ic, 4), "start_newton": (ic, 5),
             "hmin": (rc, 0), "hmax": (rc, 1), "hstart": (rc, 2), "facmin": (rc, 3),
             "facmax": (rc, 4), "facrej": (rc, 5), "facsafe": (rc, 6), "theta_min": (rc, 7),
             "newton_tol": (rc, 8), "qmin": (rc, 9), "qmax": (rc, 10)}
    for k, v in kw.items():
        arr, i = slots[k]
        arr[i] = v
    return ic, rc


CASES = ([(f"method_{k}", dict(method=k), None) for k in (0, 1, 2, 3, 4, 5, 7)] + [
    ("max_steps_3", dict(max_steps=3), None),
    ("neg_max_steps", dict(max_steps=-1), None),
    ("newton_maxit_1", dict(newton_maxit=1), None),
    ("newton_maxit_1_4a", dict(method=4, newton_maxit=1), None),
    ("newton_start_zero", dict(start_newton=1), None),
    ("neg_hmin", dict(hmin=-1.0), None),
    ("neg_hmax", dict(hmax=-1.0), None),
    ("hstart", dict(hstart=10.0), None),
    ("neg_facmin", dict(facmin=-0.5), None),
    ("facmax_2", dict(facmax=2.0), None),
    ("theta_min_neg", dict(theta_min=-1.0), None),
    ("theta_min_2", dict(theta_min=2.0), None),
    ("newton_tol_big", dict(newton_tol=2.0), None),
    ("qmin_qmax", dict(qmin=0.5, qmax=2.0), None),
    ("tiny_rtol", dict(), (1.0, 1e-17)),
    ("zero_atol", dict(), (0.0, 1e-3)),
    ("tiny_hmax", dict(hmax=1e-300), None),
    ("vector_tol", dict(scalar_tol=False), "vector"),
])


def _host_lib(mech, tmp_path):
    hdr = REPO / "kpp_b200" / "_gen" / f"{mech}.cuh"
    if not hdr.exists():
        pytest.skip("generated mechanism code not present (run the build)")
    out = tmp_path / f"host_sdirk_{mech}.so"
    # -O without FMA contraction on x86-64: the reference's own flags
    subprocess.run([shutil.which("g++"), "-O", "-fPIC", "-shared", "-std=c++17",
                    "-I", str(REPO / "kpp_b200" / "csrc"), f'-DKPP_MECH_HEADER="{hdr}"',
                    str(REPO / "tests" / "host_sdirk.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.host_sdirk_integrate.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 14
    return lib


def _host_integrate(lib, var, fix, temp, t0, t1, atol, rtol, ic, rc, cfactor, sun):
    f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
    var = f64(var).copy()
    n = var.shape[1]
    ist, rst, ierr = np.zeros((8, n), np.int32), np.zeros((3, n)), np.zeros(n, np.int32)
    args = [f64(fix), f64(temp), f64(cfactor), f64(sun), f64(t0), f64(t1), f64(atol), f64(rtol),
            np.asarray(ic, np.int32), np.asarray(rc, np.float64)]
    lib.host_sdirk_integrate(n, n, _p(var), *[_p(a) for a in args], _p(ist), _p(rst), _p(ierr))
    return var, ist, rst, ierr


@pytest.mark.skipif(not ensure_built(), reason="oracle libraries not built")
@pytest.mark.parametrize("mech", list(MECHS))
def test_sdirk_restatement_bit_identical_to_reference(mech, tmp_path):
    if not sdirk_lib_path(mech).exists():
        pytest.skip("SDIRK oracle library not present")
    if mech == "mcm_isoprene":
        from kpp_b200 import build
        if not build.library_path(mech).exists():
            pytest.skip("mcm_isoprene is built on request")
    lib = _host_lib(mech, tmp_path)
    o = SdirkOracle(mech)
    ref = OracleLib(mech)

    class Model:  # what the workload builder reads of a mechanism
        nvar = o.nvar
        species = ref.species

        @staticmethod
        def initial_values():
            return ref.initial_values()

    n = MECHS[mech]
    wl = workloads.for_mechanism(Model, mech, n, seed=11)
    fix = wl.fix if wl.fix.shape[0] else np.zeros((1, n))  # the C model pads NFIX
    steps = (0, 3) if mech == "small_strato" else (0,)
    cases = CASES if mech == "small_strato" else [c for c in CASES if c[0].startswith("method")
                                                  or c[0] in ("newton_maxit_1", "vector_tol")]
    checked = 0
    for name, ctl, tol in cases:
        ic, rc = _controls(**ctl)
        if tol == "vector":
            atol, rtol = np.linspace(0.5, 2.0, o.nvar), np.linspace(1e-4, 1e-3, o.nvar)
        elif tol is not None:
            atol, rtol = np.array([tol[0]]), np.array([tol[1]])
        else:
            atol, rtol = wl.atol, wl.rtol
        for step in steps:
            t0, t1 = wl.step_bounds(step)
            want = o.integrate(wl.var, fix, wl.temp, t0, t1, atol, rtol, ic, rc,
                               cfactor=wl.cfactor, sun=wl.sun)
            got = _host_integrate(lib, wl.var, fix, wl.temp, t0, t1, atol, rtol, ic, rc,
                                  wl.cfactor, wl.sun)
            for what, g, w in zip(("var", "istatus", "rstatus", "ierr"), got, want):
                np.testing.assert_array_equal(g, w, err_msg=f"{mech} {name} step {step}: {what}")
            checked += 1
    assert checked == len(cases) * len(steps)
