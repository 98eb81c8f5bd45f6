"""kppcu, the mechanism compiler (CPU).

  * species order and sparse LU pattern equal the reference generator's, for
    the benchmark mechanisms (golden structure) and for small mechanisms
    written here that exercise the language (comments, coefficients, hv,
    fixed species, #SETFIX, number rates, repeated reactants), by running the
    reference generator built from its sources next to kppcu;
  * the emitted device code, compiled for the host, computes the rates, Fun,
    Jac_SP, LU factorisation and solves bit for bit like the reference's own
    generated C functions (same compiler, same libm).
"""
import ctypes
import json
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle_lib import OracleLib, REPO, ensure_built, kpp_home

BUILD = REPO / "kpp_b200" / "_build"
KPP_HOME = kpp_home()
HAVE_SOURCES = (Path(KPP_HOME) / "models" / "small_strato.eqn").exists()
MECHS = ["small_strato", "saprc99"]


@pytest.fixture(scope="module")
def kppcu():
    from kpp_b200 import build
    return build.build_kppcu()


def run_kppcu(exe, kpp_file, out_prefix, home=KPP_HOME):
    r = subprocess.run([str(exe), str(kpp_file), "-o", str(out_prefix), "--home", home],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.loads(Path(str(out_prefix) + ".json").read_text())


@pytest.mark.skipif(not HAVE_SOURCES, reason="mechanism sources not present")
@pytest.mark.parametrize("mech", MECHS)
def test_structure_matches_reference_golden(kppcu, mech, tmp_path, golden_dir):
    got = run_kppcu(kppcu, REPO / "kpp_b200" / "mechanisms" / f"{mech}.kpp", tmp_path / mech)
    g = json.loads((golden_dir / f"structure_{mech}.json").read_text())
    assert got["species"] == g["species"]
    for k in ("nvar", "nfix", "nreact", "lu_nonzero"):
        assert got[k] == g[k], k
    for k in ("lu_irow", "lu_icol", "lu_crow", "lu_diag"):
        assert got[k] == g[k], k


HAVE_MCM = (Path(KPP_HOME) / "examples" / "mcm" / "mcm_isoprene.eqn").exists()


@pytest.mark.skipif(not HAVE_MCM, reason="MCM example sources not present")
def test_mcm_translation_structure_matches_reference_golden(kppcu, tmp_path, golden_dir):
    """MCM isoprene through the Fortran-to-C translation and kppcu: species
    order and LU pattern of the reference generator run on the same file."""
    from kpp_b200.gen import mcm
    mcm.write(Path(KPP_HOME), tmp_path)
    shutil.copy(REPO / "kpp_b200" / "mechanisms" / "mcm_isoprene.kpp", tmp_path)
    got = run_kppcu(kppcu, tmp_path / "mcm_isoprene.kpp", tmp_path / "out")
    g = json.loads((golden_dir / "structure_mcm_isoprene.json").read_text())
    assert got["species"] == g["species"]
    for k in ("nvar", "nfix", "nreact", "lu_nonzero", "lu_irow", "lu_icol", "lu_crow", "lu_diag"):
        assert got[k] == g[k], k


# Small mechanisms in the KPP language exercising the front end.
SMALL = {
    "toy_chain": """
#INCLUDE atoms.kpp
#DEFVAR
 A = IGNORE; B = IGNORE; C = IGNORE; D = IGNORE;
#DEFFIX
 M = IGNORE; { a comment } H2O = IGNORE;
#EQUATIONS
<r1> A + hv = 2B        : 1.0e-3*SUN;
<r2> B + B = C          : 2.5e-11;
<r3> C + M = A + D      : ARR_ab( 1.0e-12 , -300.0 );
<r4> D + H2O = 0.5A + 0.5B : (3.0E-15);
<r5> A + C = B          : 4.0e-12 ;
""",
    "toy_setfix": """
#INCLUDE atoms.kpp
#DEFVAR
 X1 = IGNORE; X2 = IGNORE; X3 = IGNORE; X4 = IGNORE; X5 = IGNORE; Y = IGNORE;
#DEFFIX
 Z = IGNORE;
#SETFIX Y;
#EQUATIONS
 X1 + X2 = X3            : 1.e-10;
 X3 + Y = X4 + X1        : 2.0e-12*TEMP;
 X4 = X5 + X2            : 0.33;
 X5 + X1 + Z = X2 + X3   : 1.5e-30;
 X2 + X5 = 2 X1          : 7.7e-13 // trailing comment
 ;
 X3 + X4 = X5            : 1.0e-11;
""",
}


@pytest.mark.skipif(not HAVE_SOURCES, reason="mechanism sources not present")
@pytest.mark.skipif(not (REPO / "oracle" / "_ref" / "kpp").exists() and not ensure_built(),
                    reason="reference generator not built")
@pytest.mark.parametrize("name", sorted(SMALL))
def test_small_mechanisms_match_reference_generator(kppcu, name, tmp_path):
    eqn = tmp_path / f"{name}.eqn"
    eqn.write_text(SMALL[name])
    # kppcu input
    (tmp_path / f"{name}_cu.kpp").write_text(f"#INCLUDE {name}.eqn\n#LANGUAGE CUDA\n")
    got = run_kppcu(kppcu, tmp_path / f"{name}_cu.kpp", tmp_path / f"{name}_cu")
    # reference generator on the same equations, C language
    (tmp_path / f"{name}.kpp").write_text(
        f"#INCLUDE {name}.eqn\n#LANGUAGE C\n#INTEGRATOR rosenbrock\n#DRIVER general\n")
    r = subprocess.run([str(REPO / "oracle" / "_ref" / "kpp"), f"{name}.kpp"], cwd=tmp_path,
                       env={**os.environ, "KPP_HOME": KPP_HOME}, capture_output=True, text=True)
    assert r.returncode in (0, 5), r.stdout[-2000:]
    par = (tmp_path / f"{name}_Parameters.h").read_text()
    ind = sorted(((int(v), n) for n, v in
                  (line.split()[1:3] for line in par.splitlines() if line.startswith("#define ind_"))))
    assert [n[4:] for _, n in ind] == got["species"]
    sp = (tmp_path / f"{name}_JacobianSP.c").read_text()

    def arr(nm):
        body = sp.split(nm + "[] = {")[1].split("}")[0]
        return [int(x) for x in body.replace("\n", " ").split(",") if x.strip()]

    assert arr("LU_ICOL") == got["lu_icol"]
    assert arr("LU_CROW") == got["lu_crow"]
    assert arr("LU_DIAG") == got["lu_diag"]


# --- emitted arithmetic, compiled for the host -------------------------------
def _host_lib(mech, tmp_path):
    hdr = REPO / "kpp_b200" / "_gen" / f"{mech}.cuh"
    if not hdr.exists():
        pytest.skip("generated mechanism code not present (run the build)")
    cxx = shutil.which("g++")
    out = tmp_path / f"host_{mech}.so"
    # -O without FMA contraction on x86-64: the reference's own flags
    adj = REPO / "kpp_b200" / "_gen" / f"{mech}_adj.cuh"
    extra = [f'-DKPP_ADJ_HEADER="{adj}"'] if adj.exists() else []
    subprocess.run([cxx, "-O", "-fPIC", "-shared", "-std=c++17", "-I", str(REPO / "kpp_b200" / "csrc"),
                    f'-DKPP_MECH_HEADER="{hdr}"', *extra, str(REPO / "tests" / "host_harness.cpp"),
                    "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.host_rates.argtypes = [ctypes.c_double] * 4 + [ctypes.c_void_p] * 3
    lib.host_fun.argtypes = [ctypes.c_void_p] * 4
    lib.host_jac.argtypes = [ctypes.c_void_p] * 4
    lib.host_decomp.argtypes = [ctypes.c_void_p]
    lib.host_solve.argtypes = [ctypes.c_void_p] * 2
    return lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


@pytest.mark.skipif(not ensure_built(), reason="oracle libraries not built")
@pytest.mark.parametrize("mech", MECHS + ["mcm_isoprene"])
def test_emitted_arithmetic_bit_identical_on_host(mech, tmp_path, golden_dir):
    h = _host_lib(mech, tmp_path)
    o = OracleLib(mech)
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    for c in range(g["var"].shape[1]):
        var = np.ascontiguousarray(g["var"][:, c])
        fix = np.ascontiguousarray(g["fix"][:, c])
        rc, vd, jv = np.zeros(o.nreact), np.zeros(o.nvar), np.zeros(o.lu_nonzero)
        h.host_rates(g["temp"][c], g["cfactor"][c], g["sun"][c], g["time"][c], _p(var), _p(fix), _p(rc))
        h.host_fun(_p(var), _p(fix), _p(rc), _p(vd))
        h.host_jac(_p(var), _p(fix), _p(rc), _p(jv))
        np.testing.assert_array_equal(rc, g["rconst"][:, c])
        np.testing.assert_array_equal(vd, g["vdot"][:, c])
        np.testing.assert_array_equal(jv, g["jvs"][:, c])
    # LU and solve against the reference's KppDecomp / KppSolve
    o.lib.KppDecomp.argtypes = [ctypes.c_void_p]
    o.lib.KppSolve.argtypes = [ctypes.c_void_p] * 2
    irow, icol, crow, diag = o.lu_pattern()
    rng = np.random.default_rng(1)
    for c in range(g["var"].shape[1]):
        m = np.ascontiguousarray(-g["jvs"][:, c])
        m[diag[:-1]] += 1.0 / (0.5 * rng.uniform(1.0, 600.0))
        a, b = m.copy(), m.copy()
        assert h.host_decomp(_p(a)) == o.lib.KppDecomp(_p(b))
        np.testing.assert_array_equal(a, b)
        x = rng.standard_normal(o.nvar)
        xa, xb = x.copy(), x.copy()
        h.host_solve(_p(a), _p(xa))
        o.lib.KppSolve(_p(b), _p(xb))
        np.testing.assert_array_equal(xa, xb)


def test_rate_classes_are_reported(tmp_path):
    hdr = REPO / "kpp_b200" / "_gen" / "saprc99.cuh"
    if not hdr.exists():
        pytest.skip("generated mechanism code not present")
    text = hdr.read_text()
    assert "#define KPP_RATES_DYNAMIC 0" in text
    assert "#define KPP_RATES_SUN 30" in text


@pytest.mark.skipif(not ensure_built(), reason="oracle libraries not built")
@pytest.mark.parametrize("mech", MECHS + ["mcm_isoprene"])
def test_adjoint_building_blocks_bit_identical_on_host(mech, tmp_path, golden_dir):
    """Jac_SP_Vec, JacTR_SP_Vec and KppSolveTR (src/gen.c:1763-1880,
    2036-2120), as kppcu emits them (<mech>_adj.cuh) and compiled for the
    host, against the reference's generated functions: bit for bit, on the
    golden Jacobians and on their factorised Rosenbrock matrices."""
    if not (REPO / "kpp_b200" / "_gen" / f"{mech}_adj.cuh").exists():
        pytest.skip("generated adjoint header not present (run the build)")
    h = _host_lib(mech, tmp_path)
    for nm in ("host_jac_sp_vec", "host_jactr_sp_vec", "host_solve_tr"):
        getattr(h, nm).argtypes = [ctypes.c_void_p] * 3
    o = OracleLib(mech)
    ref = o.lib
    for nm in ("Jac_SP_Vec", "JacTR_SP_Vec", "KppSolveTR"):
        getattr(ref, nm).argtypes = [ctypes.c_void_p] * 3
    ref.KppDecomp.argtypes = [ctypes.c_void_p]
    diag = o.lu_pattern()[3][: o.nvar]
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    rng = np.random.default_rng(9)
    for c in range(g["jvs"].shape[1]):
        jvs = np.ascontiguousarray(g["jvs"][:, c])
        uv = rng.standard_normal(o.nvar)
        for host_fn, ref_fn in ((h.host_jac_sp_vec, ref.Jac_SP_Vec),
                                (h.host_jactr_sp_vec, ref.JacTR_SP_Vec)):
            a, b = np.zeros(o.nvar), np.zeros(o.nvar)
            host_fn(_p(jvs), _p(uv), _p(a))
            ref_fn(_p(jvs), _p(uv), _p(b))
            np.testing.assert_array_equal(a, b)
        # the factorised Rosenbrock matrix 1/(h gamma) - J, then the solve
        e = -jvs.copy()
        e[diag] += 1.0 / (10.0 * 0.5)
        if ref.KppDecomp(_p(e)) != 0:
            continue
        x = rng.standard_normal(o.nvar)
        a, b = np.zeros(o.nvar), np.zeros(o.nvar)
        h.host_solve_tr(_p(e), _p(x), _p(a))
        ref.KppSolveTR(_p(e), _p(x), _p(b))
        np.testing.assert_array_equal(a, b)
