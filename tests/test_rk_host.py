"""The Runge-Kutta integrator of kpp_b200 (kpp_rk.cuh) and the generated
complex LU (<mech>_cmplx.cuh), compiled for the host, against the
reference's own C RungeKutta (int/runge_kutta.c) and KppDecompCmplxR /
KppSolveCmplxR (util/sutil.c:28-90) on the same mechanism: bit for bit, for
every method, both error estimators, the parameter error codes and the
controls, in one process.

Both sides run on the CPU with the same compiler and libm, so any difference
is an error of the restatement.  Lobatto-3A, which the reference's C
translation runs through the 3-stage formulas, only finishes short windows
(its step size collapses on longer ones: the reference then does not
return), so it is compared on those.
"""
import ctypes
import shutil
import subprocess

import numpy as np
import pytest

from kpp_b200 import workloads
from oracle_lib import REPO, OracleLib, RkOracle, _p, ensure_built, rk_lib_path


def rk_controls(method=0, scalar_tol=True, sdirk_error=1, **kw):
    """ICNTRL / RCNTRL of int/runge_kutta.c (ICNTRL[1] = 0 vector
    tolerances, [2] method, [3] max steps, [4] Newton iterations, [5] zero
    Newton start, [9] SDIRK error estimator, [10] classic controller;
    RCNTRL[0..10] Hmin, Hmax, Hstart, FacMin, FacMax, FacRej, FacSafe,
    ThetaMin, NewtonTol, Qmin, Qmax)."""
    ic, rc = [0] * 20, [0.0] * 20
    ic[1] = 1 if scalar_tol else 0
    ic[2] = method
    ic[9] = sdirk_error
    slots = {"max_steps": (ic, 3), "newton_maxit": (ic, 4), "start_newton": (ic, 5),
             "classic_controller": (ic, 10), "hmin": (rc, 0), "hmax": (rc, 1),
             "hstart": (rc, 2), "facmin": (rc, 3), "facmax": (rc, 4), "facrej": (rc, 5),
             "facsafe": (rc, 6), "theta_min": (rc, 7), "newton_tol": (rc, 8), "qmin": (rc, 9),
             "qmax": (rc, 10)}
    for k, v in kw.items():
        arr, i = slots[k]
        arr[i] = v
    return ic, rc


# (name, controls, window length in s or None for the workload's step)
CASES = ([(f"method_{m}_sdirk_err_{e}", dict(method=m, sdirk_error=e), None)
          for m in (0, 1, 2, 3, 4) for e in (1, 0)] + [
    ("lobatto3a_sdirk_err", dict(method=5), 1e-6),
    ("lobatto3a_classic_err", dict(method=5, sdirk_error=0), 1e-4),
    ("bad_method", dict(method=9), None),
    ("classic_controller", dict(classic_controller=1), None),
    ("newton_maxit_1", dict(newton_maxit=1), None),
    ("newton_maxit_2", dict(newton_maxit=2), None),
    ("newton_start_zero", dict(start_newton=1), None),
    ("hstart", dict(hstart=10.0), None),
    ("hmin", dict(hmin=1.0), None),
    ("hmax", dict(hmax=50.0), None),
    ("max_steps_3", dict(max_steps=3), None),
    ("neg_max_steps", dict(max_steps=-1), None),
    ("neg_newton_maxit", dict(newton_maxit=-2), None),
    ("facmax_below_1", dict(facmax=0.5), None),
    ("theta_min_2", dict(theta_min=2.0), None),
    ("newton_tol_tiny", dict(newton_tol=1e-17), None),
    ("qmin_2", dict(qmin=2.0), None),
    ("theta_min_half", dict(theta_min=0.5), None),
    ("qmin_qmax", dict(qmin=0.5, qmax=2.0), None),
    ("vector_tol", dict(scalar_tol=False), None),
    ("tiny_rtol", dict(), "tiny_rtol"),
])

MECHS = {"small_strato": (64, (0, 3), None), "saprc99": (8, (0,), "methods"),
         "mcm_isoprene": (4, (0,), "methods")}


def _host_lib(mech, tmp_path):
    gen = REPO / "kpp_b200" / "_gen"
    hdr, cmplx = gen / f"{mech}.cuh", gen / f"{mech}_cmplx.cuh"
    if not (hdr.exists() and cmplx.exists()):
        pytest.skip("generated mechanism code not present (run the build)")
    out = tmp_path / f"host_rk_{mech}.so"
    # -O without FMA contraction on x86-64: the reference's own flags
    subprocess.run([shutil.which("g++"), "-O", "-fPIC", "-shared", "-std=c++17",
                    "-I", str(REPO / "kpp_b200" / "csrc"), f'-DKPP_MECH_HEADER="{hdr}"',
                    f'-DKPP_CMPLX_HEADER="{cmplx}"', str(REPO / "tests" / "host_rk.cpp"),
                    "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.host_rk_integrate.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 14
    lib.host_decomp_cmplx.argtypes = [ctypes.c_void_p] * 2
    lib.host_solve_cmplx.argtypes = [ctypes.c_void_p] * 4
    return lib


def _host_integrate(lib, var, fix, temp, t0, t1, atol, rtol, ic, rc, cfactor, sun):
    f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
    var = f64(var).copy()
    n = var.shape[1]
    ist, rst, ierr = np.zeros((8, n), np.int32), np.zeros((3, n)), np.zeros(n, np.int32)
    args = [f64(fix), f64(temp), f64(cfactor), f64(sun), f64(t0), f64(t1), f64(atol), f64(rtol),
            np.asarray(ic, np.int32), np.asarray(rc, np.float64)]
    lib.host_rk_integrate(n, n, _p(var), *[_p(a) for a in args], _p(ist), _p(rst), _p(ierr))
    return var, ist, rst, ierr


def _model(mech):
    o, ref = RkOracle(mech), OracleLib(mech)

    class Model:  # what the workload builder reads of a mechanism
        nvar = o.nvar
        species = ref.species

        @staticmethod
        def initial_values():
            return ref.initial_values()

    return o, ref, Model


@pytest.mark.skipif(not ensure_built(), reason="oracle libraries not built")
@pytest.mark.parametrize("mech", list(MECHS))
def test_complex_lu_bit_identical_to_reference(mech, tmp_path, golden_dir):
    if not rk_lib_path(mech).exists():
        pytest.skip("Runge-Kutta oracle library not present")
    lib = _host_lib(mech, tmp_path)
    o, ref, _ = _model(mech)
    diag = ref.lu_pattern()[3][: o.nvar]
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    rng = np.random.default_rng(3)
    for c in range(g["jvs"].shape[1]):
        for h in (1e-3, 10.0, 600.0):
            jr = -g["jvs"][:, c].copy()
            ji = np.zeros_like(jr)
            jr[diag] += 2.681082873627752 / h
            ji[diag] += 3.050430199247411 / h
            a_r, a_i, b_r, b_i = jr.copy(), ji.copy(), jr.copy(), ji.copy()
            assert lib.host_decomp_cmplx(_p(b_r), _p(b_i)) == o.decomp_cmplx(a_r, a_i)
            np.testing.assert_array_equal(b_r, a_r)
            np.testing.assert_array_equal(b_i, a_i)
            xr, xi = rng.standard_normal(o.nvar), rng.standard_normal(o.nvar)
            x1r, x1i, x2r, x2i = xr.copy(), xi.copy(), xr.copy(), xi.copy()
            o.solve_cmplx(a_r, a_i, x1r, x1i)
            lib.host_solve_cmplx(_p(b_r), _p(b_i), _p(x2r), _p(x2i))
            np.testing.assert_array_equal(x2r, x1r)
            np.testing.assert_array_equal(x2i, x1i)


@pytest.mark.skipif(not ensure_built(), reason="oracle libraries not built")
@pytest.mark.parametrize("mech", list(MECHS))
def test_rk_restatement_bit_identical_to_reference(mech, tmp_path):
    if not rk_lib_path(mech).exists():
        pytest.skip("Runge-Kutta oracle library not present")
    lib = _host_lib(mech, tmp_path)
    o, _, Model = _model(mech)
    n, steps, subset = MECHS[mech]
    wl = workloads.for_mechanism(Model, mech, n, seed=11)
    fix = wl.fix if wl.fix.shape[0] else np.zeros((1, n))  # the C model pads NFIX
    cases = CASES if subset is None else [c for c in CASES if c[0].startswith("method_")]
    checked = 0
    for name, ctl, window in cases:
        ic, rc = rk_controls(**ctl)
        atol, rtol = wl.atol, wl.rtol
        if not ctl.get("scalar_tol", True):
            atol, rtol = np.linspace(0.5, 2.0, o.nvar), np.linspace(1e-4, 1e-3, o.nvar)
        if window == "tiny_rtol":
            rtol = np.array([1e-17])
        for step in steps:
            t0, t1 = wl.step_bounds(step)
            if isinstance(window, float):
                t1 = t0 + window
            want = o.integrate(wl.var, fix, wl.temp, t0, t1, atol, rtol, ic, rc,
                               cfactor=wl.cfactor, sun=wl.sun)
            got = _host_integrate(lib, wl.var, fix, wl.temp, t0, t1, atol, rtol, ic, rc,
                                  wl.cfactor, wl.sun)
            for what, gv, wv in zip(("var", "istatus", "rstatus", "ierr"), got, want):
                np.testing.assert_array_equal(gv, wv, err_msg=f"{mech} {name} step {step}: {what}")
            checked += 1
    assert checked == len(cases) * len(steps)
