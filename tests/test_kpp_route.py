"""KPP's own generator with kpp_b200's CUDA target (#LANGUAGE CUDA) (CPU).

kpp_b200/kppgen builds KPP's generator from its sources with the CUDA writer
(kpp_b200/kppgen/code_cuda.c) hooked into its language switch, and runs it on
a mechanism.  Compiled for the host (tests/host_route.cpp), the device code it
writes must compute Update_RCONST, Fun, Jac_SP, KppDecomp and KppSolve bit for
bit as the reference's own generated C does (the golden fixtures and the
oracle library), and so as the kppcu route does, on all three mechanisms.
"""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import REPO, OracleLib, kpp_home, lib_path

MECHS = ["small_strato", "saprc99", "mcm_isoprene"]
HOME = kpp_home()
pytestmark = pytest.mark.skipif(not (HOME and Path(HOME, "src", "gen.c").exists()),
                                reason="KPP sources not present")


def constant_rate_equations(mech):
    """Equations whose rate is a number (kppcu's kRateKind 0): folded into Fun
    and Jac_SP, and not written by Update_RCONST."""
    hdr = (REPO / "kpp_b200" / "_gen" / f"{mech}.cuh").read_text()
    body = re.search(r"kRateKind\[\d+\] = \{([^}]*)\}", hdr).group(1)
    kinds = np.array([int(x) for x in body.replace("\n", " ").split(",") if x.strip()])
    return kinds == 0


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.fixture(scope="module")
def route_libs(tmp_path_factory):
    from kpp_b200.kppgen import build as kppgen
    out = {}
    for mech in MECHS:
        # MCM's Hessian (not compared here) takes KPP's generator about 20
        # minutes; the functions compared are written without it
        d = kppgen.generate(mech, HOME, hessian=mech != "mcm_isoprene")
        so = tmp_path_factory.mktemp(mech) / "route.so"
        subprocess.run([shutil.which("g++"), "-O2", "-fPIC", "-shared", "-std=c++17",
                        "-I", str(REPO / "kpp_b200" / "csrc"), "-I", str(d),
                        f'-DROUTE_INCLUDES="{d / "route_includes.h"}"',
                        str(REPO / "tests" / "host_route.cpp"), "-o", str(so)], check=True)
        lib = ctypes.CDLL(str(so))
        lib.route_rates.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [ctypes.c_void_p] * 3
        for f in ("route_fun", "route_jac"):
            getattr(lib, f).argtypes = [ctypes.c_void_p] * 4
        lib.route_decomp.argtypes = [ctypes.c_void_p]
        lib.route_solve.argtypes = [ctypes.c_void_p] * 2
        out[mech] = (d, lib)
    return out


def test_generator_writes_the_cuda_target(route_libs):
    for mech, (d, _) in route_libs.items():
        for suffix in ("_Function.cu", "_Jacobian.cu", "_JacobianSP.cu", "_LinearAlgebra.cu",
                       "_Rates.cu"):
            text = (d / f"{mech}{suffix}").read_text()
            assert "__device__" in text, (mech, suffix)
        assert "Generated by KPP" in (d / f"{mech}_Function.cu").read_text()


@pytest.mark.parametrize("mech", MECHS)
def test_rates_fun_jac_bit_identical_to_reference(route_libs, mech, golden_dir):
    _, h = route_libs[mech]
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    nvar, nreact = g["var"].shape[0], g["rconst"].shape[0]
    for c in range(g["var"].shape[1]):
        var = np.ascontiguousarray(g["var"][:, c])
        fix = np.ascontiguousarray(g["fix"][:, c]) if g["fix"].shape[0] else np.zeros(1)
        rc = np.full(nreact, np.nan)
        h.route_rates(nvar, g["temp"][c], g["cfactor"][c], g["sun"][c], g["time"][c], _p(var),
                      _p(fix), _p(rc))
        # every rate except the constant ones, which the reference stores in
        # RCONST only in Initialize() and folds into Fun / Jac_SP
        const = constant_rate_equations(mech)
        # contiguous copies held for the length of each call
        rc_ref = np.ascontiguousarray(g["rconst"][:, c])
        np.testing.assert_array_equal(np.isnan(rc), const)
        np.testing.assert_array_equal(rc[~const], rc_ref[~const])
        vd, jv = np.zeros(nvar), np.zeros(g["jvs"].shape[0])
        h.route_fun(_p(var), _p(fix), _p(rc_ref), _p(vd))
        h.route_jac(_p(var), _p(fix), _p(rc_ref), _p(jv))
        np.testing.assert_array_equal(vd, g["vdot"][:, c])
        np.testing.assert_array_equal(jv, g["jvs"][:, c])


@pytest.mark.parametrize("mech", MECHS)
def test_lu_and_solve_bit_identical_to_reference(route_libs, mech, golden_dir):
    if not lib_path(mech).exists():
        pytest.skip("oracle libraries not present")
    _, h = route_libs[mech]
    o = OracleLib(mech)
    o.lib.KppDecomp.argtypes = [ctypes.c_void_p]
    o.lib.KppSolve.argtypes = [ctypes.c_void_p] * 2
    diag = o.lu_pattern()[3][:-1]
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    rng = np.random.default_rng(2)
    for c in range(g["var"].shape[1]):
        m = np.ascontiguousarray(-g["jvs"][:, c])
        m[diag] += 1.0 / (0.5 * rng.uniform(1.0, 600.0))
        a, b = m.copy(), m.copy()
        assert h.route_decomp(_p(a)) == o.lib.KppDecomp(_p(b))
        np.testing.assert_array_equal(a, b)
        x = rng.standard_normal(o.nvar)
        xa, xb = x.copy(), x.copy()
        h.route_solve(_p(a), _p(xa))
        o.lib.KppSolve(_p(b), _p(xb))
        np.testing.assert_array_equal(xa, xb)
