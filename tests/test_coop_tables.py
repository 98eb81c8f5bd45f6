"""The warp-per-cell kernel's schedules against the reference (CPU).

kppcu's tables for kpp_b200/csrc/kpp_coop.cuh, executed by the CPU emulation
in tests/coop_emulator.py exactly as the kernel's lanes execute them, must
reproduce the reference's own generated Fun, Jac_SP, KppDecomp
(util/sutil.c:2-23) and KppSolve (src/gen.c:1960-2034) bit for bit on the
golden cells: the schedules only reorder independent operations.
"""
import ctypes

import numpy as np
import pytest

from coop_emulator import CoopTables
from oracle_lib import REPO, OracleLib, lib_path

MECHS = ["small_strato", "saprc99"]


def _tables(mech):
    hdr = REPO / "kpp_b200" / "_gen" / f"{mech}.cuh"
    if not hdr.exists():
        pytest.skip("generated mechanism code not present")
    return CoopTables(hdr)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("mech", MECHS)
def test_products_and_sums_reproduce_fun_and_jac(mech, golden_dir):
    t = _tables(mech)
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    for c in range(g["var"].shape[1]):
        var, fix, rc = g["var"][:, c], g["fix"][:, c], g["rconst"][:, c]
        np.testing.assert_array_equal(np.array(t.fun(var, fix, rc)), g["vdot"][:, c])
        np.testing.assert_array_equal(np.array(t.jac(var, fix, rc)), g["jvs"][:, c])
        # the Rosenbrock matrix: -Jac with 1/(h gamma) on the diagonal
        ghinv = 1.0 / (0.5 * 37.0)
        want = -g["jvs"][:, c]
        diag = t.tab[t.O_DIAG:t.O_DIAG + t.nvar]
        want[diag] = want[diag] + ghinv
        np.testing.assert_array_equal(np.array(t.jac(var, fix, rc, neg=True, ghinv=ghinv)),
                                      want)


@pytest.mark.parametrize("mech", MECHS)
def test_lu_and_solves_reproduce_kppdecomp_and_kppsolve(mech, golden_dir):
    t = _tables(mech)
    if not lib_path(mech).exists():
        pytest.skip("oracle libraries not present")
    oracle = OracleLib(mech)
    ref = oracle.lib
    pattern = oracle.lu_pattern()
    ref.KppDecomp.argtypes = [ctypes.c_void_p]
    ref.KppSolve.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    rng = np.random.default_rng(5)
    diag = t.tab[t.O_DIAG:t.O_DIAG + t.nvar]
    checked = 0
    for c in range(g["var"].shape[1]):
        for h in (1e-3, 1.0, 600.0):
            e = -g["jvs"][:, c].copy()
            e[diag] = e[diag] + 1.0 / (h * 0.5)
            want = np.ascontiguousarray(e.copy())
            rc = ref.KppDecomp(_p(want))
            got = list(e)
            assert t.decomp(got) == rc
            if rc != 0:
                continue
            np.testing.assert_array_equal(np.array(got), want)
            x = rng.standard_normal(t.nvar)
            xw = np.ascontiguousarray(x.copy())
            ref.KppSolve(_p(want), _p(xw))
            xg = list(x)
            t.solve(got, xg, pattern)
            np.testing.assert_array_equal(np.array(xg), xw)
            checked += 1
    assert checked > 0


@pytest.mark.parametrize("mech", MECHS)
def test_zero_diagonal_is_reported_like_kppdecomp(mech, golden_dir):
    t = _tables(mech)
    if not lib_path(mech).exists():
        pytest.skip("oracle libraries not present")
    ref = OracleLib(mech).lib
    ref.KppDecomp.argtypes = [ctypes.c_void_p]
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    diag = t.tab[t.O_DIAG:t.O_DIAG + t.nvar]
    for row in (0, t.nvar // 2, t.nvar - 1):
        e = -g["jvs"][:, 0].copy()
        e[diag] = e[diag] + 2.0
        e[diag[row]] = 0.0
        want = np.ascontiguousarray(e.copy())
        assert t.decomp(list(e)) == ref.KppDecomp(_p(want)) == row + 1
