"""The C ABI (CPU): every library loads, exports every entry point that
include/kpp_b200.h declares, and describes its mechanism like the reference
(no compute calls: these run without a GPU)."""
import ctypes
import json
import re
import subprocess

import numpy as np
import pytest

from kpp_b200 import Mechanism, from_fortran, library_path, make_controls
from oracle_lib import REPO

MECHS = ["small_strato", "saprc99", "mcm_isoprene"]
HEADER = REPO / "include" / "kpp_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(kpp_b200_\w+)\s*\(", text)))


def exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def _skip_on_request(mech):
    from kpp_b200 import build
    if mech in build.ON_REQUEST and not library_path(mech).exists():
        pytest.skip(f"{mech} is built on request: python -m kpp_b200.build {mech}")


@pytest.mark.parametrize("mech", MECHS)
def test_library_exports_every_declared_entry(mech):
    _skip_on_request(mech)
    lib = library_path(mech)
    assert lib.exists(), "build the libraries first: python -m kpp_b200.build"
    names = declared_functions()
    assert "kpp_b200_rosenbrock" in names and len(names) >= 8
    missing = [n for n in names if n not in exported(lib)]
    assert not missing, missing
    ctypes.CDLL(str(lib))  # loads without a GPU


@pytest.mark.parametrize("mech", ["small_strato", "saprc99"])
def test_route_library_exports_every_declared_entry(mech):
    """The libraries built on KPP's own generator (#LANGUAGE CUDA) carry the
    same C ABI, the Rosenbrock adjoint included."""
    from kpp_b200 import build
    lib = build.library_path(mech, "kpp")
    if not lib.exists():
        pytest.skip(f"{lib.name} not built (KPP's sources were not found at build time)")
    missing = [n for n in declared_functions() if n not in exported(lib)]
    assert not missing, missing
    ctypes.CDLL(str(lib))


@pytest.mark.parametrize("mech", MECHS)
def test_mechanism_description_matches_reference(mech, golden_dir):
    _skip_on_request(mech)
    m = Mechanism(mech)
    g = json.loads((golden_dir / f"structure_{mech}.json").read_text())
    assert m.name == mech
    assert [m.nvar, m.nfix, m.nreact, m.lu_nonzero] == [g["nvar"], g["nfix"], g["nreact"], g["lu_nonzero"]]
    assert m.species == g["species"]
    irow, icol, crow, diag = m.lu_pattern()
    assert icol == g["lu_icol"] and crow == g["lu_crow"] and diag == g["lu_diag"] and irow == g["lu_irow"]


@pytest.mark.parametrize("mech", MECHS)
def test_initial_values_match_reference_initialize(mech):
    _skip_on_request(mech)
    from oracle_lib import OracleLib, ensure_built
    if not ensure_built():
        pytest.skip("oracle libraries not built")
    c, cf = Mechanism(mech).initial_values()
    rc, rcf = OracleLib(mech).initial_values()
    assert cf == rcf
    np.testing.assert_array_equal(np.array(c), rc)


def test_entry_points_reject_bad_arguments_without_gpu():
    m = Mechanism("small_strato")
    lib = m.lib
    ip = (ctypes.c_int * 20)()
    rp = (ctypes.c_double * 20)()
    # ld < ncells and null pointers fail before touching the device
    rc = lib.kpp_b200_rosenbrock(4, 2, None, None, None, None, None, None, None, None, None, ip, rp,
                                 None, None, None, None, None)
    assert rc == 1 and b"ncells" in lib.kpp_b200_last_error()
    rc = lib.kpp_b200_rosenbrock(4, 4, None, None, None, None, None, None, None, None, None, ip, rp,
                                 None, None, None, None, None)
    assert rc == 1 and b"null" in lib.kpp_b200_last_error()
    # an empty batch is a no-op
    assert lib.kpp_b200_rosenbrock(0, 0, None, None, None, None, None, None, None, None, None, ip,
                                   rp, None, None, None, None, None) == 0
    # the SDIRK entry checks the same way
    rc = lib.kpp_b200_sdirk(4, 2, None, None, None, None, None, None, None, None, None, ip, rp,
                            None, None, None, None)
    assert rc == 1 and b"ncells" in lib.kpp_b200_last_error()
    rc = lib.kpp_b200_sdirk(4, 4, None, None, None, None, None, None, None, None, None, ip, rp,
                            None, None, None, None)
    assert rc == 1 and b"null" in lib.kpp_b200_last_error()
    assert lib.kpp_b200_sdirk(0, 0, None, None, None, None, None, None, None, None, None, ip, rp,
                              None, None, None, None) == 0
    # and the Runge-Kutta entry
    rc = lib.kpp_b200_runge_kutta(4, 2, None, None, None, None, None, None, None, None, None, ip,
                                  rp, None, None, None, None)
    assert rc == 1 and b"ncells" in lib.kpp_b200_last_error()
    rc = lib.kpp_b200_runge_kutta(4, 4, None, None, None, None, None, None, None, None, None, ip,
                                  rp, None, None, None, None)
    assert rc == 1 and b"null" in lib.kpp_b200_last_error()
    assert lib.kpp_b200_runge_kutta(0, 0, None, None, None, None, None, None, None, None, None,
                                    ip, rp, None, None, None, None) == 0
    # the adjoint building blocks
    assert lib.kpp_b200_jac_vec(4, 2, None, None, None, 0, None) == 1
    assert lib.kpp_b200_jac_vec(4, 4, None, None, None, 0, None) == 1
    assert b"null" in lib.kpp_b200_last_error()
    assert lib.kpp_b200_solve_tr(4, 4, None, None, None, None) == 1
    assert lib.kpp_b200_jac_vec(0, 0, None, None, None, 1, None) == 0
    # and the host-array entries of both
    for entry in (lib.kpp_b200_sdirk_host, lib.kpp_b200_runge_kutta_host):
        rc = entry(4, 2, None, None, None, None, None, None, None, None, None, ip, rp, None, None,
                   None, 0)
        assert rc == 1 and b"ncells" in lib.kpp_b200_last_error()
        rc = entry(4, 4, None, None, None, None, None, None, None, None, None, ip, rp, None, None,
                   None, 0)
        assert rc == 1 and b"null" in lib.kpp_b200_last_error()


def test_controls_layouts():
    ipar, rpar = make_controls(method="rodas4", scalar_tol=False, max_steps=500, hmin=1e-3,
                               hmax=100.0, hstart=1.0, facmin=0.1, facmax=5.0, facrej=0.2,
                               facsafe=0.8, autonomous=True)
    assert ipar[:4] == [1, 0, 500, 5]
    assert rpar[:7] == [1e-3, 100.0, 1.0, 0.1, 5.0, 0.2, 0.8]
    icntrl = [1, 0, 5, 500] + [0] * 16   # ICNTRL(3) = method, ICNTRL(4) = max steps
    rcntrl = [1e-3, 100.0, 1.0, 0.1, 5.0, 0.2, 0.8] + [0.0] * 13
    assert from_fortran(icntrl, rcntrl) == (ipar, rpar)


def test_scheduler_library_exports_every_declared_entry():
    """libkpp_b200_sched.so exports every function of include/kpp_sched.h and
    loads without a GPU; creating a network without a GPU fails loudly."""
    from kpp_b200.build import LIB
    lib = LIB / "libkpp_b200_sched.so"
    assert lib.exists(), "build the libraries first: python -m kpp_b200.build"
    text = re.sub(r"/\*.*?\*/", "", (REPO / "include" / "kpp_sched.h").read_text(), flags=re.S)
    names = sorted(set(re.findall(r"\b(kpp_sched_\w+)\s*\(", text)))
    assert "kpp_sched_plan" in names and len(names) >= 12
    missing = [n for n in names if n not in exported(lib)]
    assert not missing, missing
    ctypes.CDLL(str(lib))
    import torch
    if not torch.cuda.is_available():
        from kpp_b200.scheduler import Mlp, SchedError
        with pytest.raises(SchedError):
            Mlp(10)


@pytest.mark.parametrize("mech", MECHS)
def test_user_species_map_matches_reference_shuffle(mech):
    """kpp_b200_user_species against the reference's own generated
    Shuffle_user2kpp / Shuffle_kpp2user (src/gen.c:3401-3468)."""
    _skip_on_request(mech)
    from oracle_lib import OracleLib, ensure_built
    if not ensure_built():
        pytest.skip("oracle libraries not built")
    o = OracleLib(mech)
    idx = Mechanism(mech).user_species()
    nuser = len(idx)
    v_user = (np.arange(nuser) + 1.0).astype(np.float64)
    v = np.full(o.nvar, -1.0)
    o.lib.Shuffle_user2kpp.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    o.lib.Shuffle_user2kpp(ctypes.c_void_p(v_user.ctypes.data), ctypes.c_void_p(v.ctypes.data))
    want = np.full(o.nvar, -1.0)
    for k, f in enumerate(idx):
        if f >= 0:
            want[f] = v_user[k]
    np.testing.assert_array_equal(v, want)
    back = np.full(nuser, -7.0)
    o.lib.Shuffle_kpp2user.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    o.lib.Shuffle_kpp2user(ctypes.c_void_p(v.ctypes.data), ctypes.c_void_p(back.ctypes.data))
    got = np.array([v_user[k] if f >= 0 else -7.0 for k, f in enumerate(idx)])
    np.testing.assert_array_equal(back, got)
