"""The Rosenbrock discrete adjoint (kpp_b200/csrc/kpp_adj_int.cuh) against the
reference's own RosenbrockADJ (int/rosenbrock_adj.c) (CPU).

The adjoint runs on the device code that KPP's own generator writes with
#LANGUAGE CUDA and #HESSIAN ON (kpp_b200/kppgen); compiled for the host
(tests/host_adj.cpp, host libm and the C library's pow, as the reference
calls it), it must give the reference's results bit for bit: the final
state, the NADJ adjoint vectors Lambda, ISTATUS[1..8], RSTATUS[1..3] and
IERR, for every method the reference selects (ICNTRL[2] = 0..5 and 7), one
to three adjoints, time-dependent and autonomous runs, scalar and vector
tolerances, saved and recomputed factorisations (ICNTRL[7]), the forward
pass alone (ICNTRL[6] = 1) and every error return.  The reference is the
mechanism generated with #INTEGRATOR rosenbrock_adj and driven cell by cell
(oracle/refkpp/batch_driver_adj.c).
"""
import ctypes
import shutil
import subprocess

import numpy as np
import pytest

from oracle_lib import REF_DIR, REPO, OracleLib, kpp_home

HOME = kpp_home()
MECHS = ["small_strato", "saprc99"]
BUFSIZE = 5000


def adj_lib_path(mech):
    return REF_DIR / f"{mech}_adj" / f"libkppadj_{mech}.so"


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


_SIG = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 9 + [ctypes.c_int, ctypes.c_void_p,
                                                                ctypes.c_void_p, ctypes.c_void_p,
                                                                ctypes.c_int] + [ctypes.c_void_p] * 3


@pytest.fixture(scope="module")
def libs(tmp_path_factory):
    if not (HOME and (REPO / "kpp_b200" / "_gen" / "saprc99.cuh").exists()):
        pytest.skip("KPP sources or generated mechanism code not present")
    from kpp_b200.kppgen import build as kppgen
    out = {}
    for mech in MECHS:
        if not adj_lib_path(mech).exists():
            pytest.skip("adjoint oracle libraries not present")
        d = kppgen.generate(mech, HOME)
        so = tmp_path_factory.mktemp(mech) / "adj.so"
        gen = REPO / "kpp_b200" / "_gen"
        subprocess.run([shutil.which("g++"), "-O", "-fPIC", "-shared", "-std=c++17",
                        "-I", str(REPO / "kpp_b200" / "csrc"), "-I", str(REPO / "kpp_b200" / "kppgen"),
                        "-I", str(d), "-I", str(gen), f'-DKPP_MECH_HEADER="{gen / (mech + ".cuh")}"',
                        f'-DROUTE_INCLUDES="{d / "route_includes.h"}"',
                        str(REPO / "tests" / "host_adj.cpp"), "-o", str(so)], check=True)
        host = ctypes.CDLL(str(so))
        host.host_adj_integrate.argtypes = _SIG
        ref = ctypes.CDLL(str(adj_lib_path(mech)))
        ref.kppadj_integrate.argtypes = _SIG
        out[mech] = (host.host_adj_integrate, ref.kppadj_integrate)
    return out


def run(fn, wl, nadj, icntrl, rcntrl, atol, rtol, lam0, bufsize=BUFSIZE):
    n = wl.ncells
    var = np.ascontiguousarray(wl.var).copy()
    fix = np.ascontiguousarray(wl.fix) if wl.fix.shape[0] else np.zeros((1, n))
    lam = lam0.copy()
    t0, t1 = wl.step_bounds(0)
    ist = np.zeros((8, n), np.int32)
    rst = np.zeros((3, n))
    ierr = np.zeros(n, np.int32)
    f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
    cf, sun = f64(wl.cfactor), f64(wl.sun)
    ic = np.ascontiguousarray(icntrl, dtype=np.int32)
    rc = np.ascontiguousarray(rcntrl, dtype=np.float64)
    at, rt = f64(atol), f64(rtol)
    temp, t0, t1 = f64(wl.temp), f64(t0), f64(t1)
    from oracle_lib import quiet_stdout
    with quiet_stdout():
        fn(n, n, _p(var), _p(fix), _p(temp), _p(cf), _p(sun), _p(t0), _p(t1), _p(at), _p(rt),
           nadj, _p(lam), _p(ic), _p(rc), bufsize, _p(ist), _p(rst), _p(ierr))
    return var, lam, ist, rst, ierr


def controls(method=0, autonomous=False, vector=False, save_lu=False, adjoint=0, **kw):
    ic, rc = [0] * 20, [0.0] * 20
    ic[0] = 1 if autonomous else 0
    ic[1] = 0 if vector else 1
    ic[2] = method
    ic[6] = adjoint
    ic[7] = 1 if save_lu else 0
    for key, val in kw.items():
        slot = {"max_steps": (ic, 3), "cadj": (ic, 5), "hmin": (rc, 0), "hmax": (rc, 1),
                "hstart": (rc, 2), "facmin": (rc, 3), "facmax": (rc, 4), "facrej": (rc, 5),
                "facsafe": (rc, 6)}[key]
        slot[0][slot[1]] = val
    return ic, rc


def check(libs, mech, ncells, seed, nadj, ic, rc, vector=False, bufsize=BUFSIZE):
    from kpp_b200 import workloads
    host, ref = libs[mech]
    wl = workloads.for_mechanism(OracleLib(mech), mech, ncells, seed=seed)
    nvar = wl.var.shape[0]
    atol = np.linspace(1e-2, 1.0, nvar) if vector else wl.atol
    rtol = np.linspace(1e-4, 1e-3, nvar) if vector else wl.rtol
    lam0 = np.random.default_rng(seed).standard_normal((max(nadj, 1) * nvar, ncells))
    a = run(host, wl, nadj, ic, rc, atol, rtol, lam0, bufsize)
    b = run(ref, wl, nadj, ic, rc, atol, rtol, lam0, bufsize)
    for x, y, nm in zip(a, b, ("var", "lambda", "istatus", "rstatus", "ierr")):
        np.testing.assert_array_equal(x, y, err_msg=f"{mech}: {nm}")
    return b


@pytest.mark.parametrize("mech", MECHS)
@pytest.mark.parametrize("method", [0, 1, 2, 3, 4, 5, 7])
def test_every_method_bit_identical(libs, mech, method):
    ic, rc = controls(method=method)
    var, lam, ist, rst, ierr = check(libs, mech, 12, 31 + method, 2, ic, rc)
    assert (ierr == 1).all()
    assert (ist[2] > 1).all()  # several steps, so the backward pass ran


@pytest.mark.parametrize("mech", MECHS)
@pytest.mark.parametrize("case", ["autonomous", "vector_tol", "save_lu", "one_adjoint",
                                  "three_adjoints", "forward_only", "hstart_hmax"])
def test_options_bit_identical(libs, mech, case):
    kw = {"autonomous": dict(autonomous=True), "vector_tol": dict(vector=True),
          "save_lu": dict(save_lu=True), "one_adjoint": {}, "three_adjoints": {},
          "forward_only": dict(adjoint=1), "hstart_hmax": dict(hstart=1.0, hmax=100.0)}[case]
    nadj = {"one_adjoint": 1, "three_adjoints": 3}.get(case, 2)
    vector = kw.pop("vector", False)
    ic, rc = controls(method=5 if case == "save_lu" else 0, vector=vector, **kw)
    _, _, _, _, ierr = check(libs, mech, 10, 41, nadj, ic, rc, vector=vector)
    assert (ierr == 1).all()


@pytest.mark.parametrize("case,code", [("max_steps_given", -1), ("bad_method", -2),
                                       ("bad_cadj", -2), ("bad_adjoint_type", -9),
                                       ("neg_hmin", -3), ("neg_hstart", -3), ("neg_facmax", -4),
                                       ("tiny_buffer", -6)])
def test_error_returns_bit_identical(libs, case, code):
    kw = {"max_steps_given": dict(max_steps=50), "bad_method": dict(method=6),
          "bad_cadj": dict(cadj=9), "bad_adjoint_type": dict(adjoint=5),
          "neg_hmin": dict(hmin=-1.0), "neg_hstart": dict(hstart=-1.0),
          "neg_facmax": dict(facmax=-2.0), "tiny_buffer": {}}[case]
    ic, rc = controls(**kw)
    _, _, _, _, ierr = check(libs, "small_strato", 6, 51, 2, ic, rc,
                             bufsize=4 if case == "tiny_buffer" else BUFSIZE)
    assert (ierr == code).all()
