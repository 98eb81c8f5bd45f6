"""ctypes access to the oracle libraries (test infrastructure only).

oracle/_ref/<mech>/libkppref_<mech>.so holds the reference's own
KPP-generated C model for <mech> with
  kppref_integrate  the reference Rosenbrock (int/rosenbrock.c) driven per
                    cell by oracle/refkpp/batch_driver.c
  kppor_integrate   the CPU restatement oracle/ros_oracle.c
  kppref_fun_jac    the generated Update_RCONST / Fun / Jac_SP of one cell
Both integrate entries take numpy arrays in the ABI layout ([rows, ld],
cell index fastest).
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
REF_DIR = REPO / "oracle" / "_ref"
_vp = ctypes.c_void_p


def kpp_home() -> str:
    """KPP's source tree: $KPP_HOME, else the tree the oracle was last built
    from (recorded by oracle/build_ref.sh), else empty."""
    home = os.environ.get("KPP_HOME", "")
    if home:
        return home
    rec = REF_DIR / "kpp_home"
    return rec.read_text().strip() if rec.exists() else ""


def lib_path(mech: str, opt: str = "") -> Path:
    return REF_DIR / mech / f"libkppref_{mech}{opt}.so"


def ensure_built(mechs=("small_strato", "saprc99", "mcm_isoprene")) -> bool:
    """Build the oracle when its libraries are missing and the reference
    sources are present; True when every library exists afterwards."""
    if all(lib_path(m).exists() for m in mechs):
        return True
    script = REPO / "oracle" / "build_ref.sh"
    subprocess.run(["bash", str(script), *mechs], check=False,
                   stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return all(lib_path(m).exists() for m in mechs)


def _p(a):
    return None if a is None else _vp(a.ctypes.data)


class OracleLib:
    def __init__(self, mech: str, opt: str = ""):
        self.mech = mech
        self.lib = ctypes.CDLL(str(lib_path(mech, opt)))
        d = (ctypes.c_int * 5)()
        self.lib.kppref_dims(d)
        self.nvar, self.nfix, self.nspec, self.nreact, self.lu_nonzero = list(d)
        self.lib.kppref_species_name.restype = ctypes.c_char_p
        self.species = [self.lib.kppref_species_name(i).decode() for i in range(self.nspec)]
        for fn in ("kppref_integrate", "kppor_integrate"):
            getattr(self.lib, fn).argtypes = [ctypes.c_int, ctypes.c_int] + [_vp] * 15
        self.lib.kppref_fun_jac.argtypes = [_vp, _vp, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, _vp, _vp, _vp]

    def initial_values(self):
        c = np.zeros(self.nspec)
        cf = ctypes.c_double()
        self.lib.kppref_initial_values(_p(c), ctypes.byref(cf))
        return c, cf.value

    def lu_pattern(self):
        n, nz = self.nvar, self.lu_nonzero
        irow, icol = np.zeros(nz, np.int32), np.zeros(nz, np.int32)
        crow, diag = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
        self.lib.kppref_lu_pattern(_p(irow), _p(icol), _p(crow), _p(diag))
        return irow, icol, crow, diag

    def integrate(self, var, fix, temp, tstart, tend, atol, rtol, ipar, rpar, cfactor=None,
                  sun=None, hstart=None, which="ref"):
        """Integrate every cell; returns (var_out, istatus, rstatus, ierr)."""
        var = np.ascontiguousarray(var, dtype=np.float64).copy()
        ld = var.shape[1]
        f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        fix, temp, tstart, tend = f64(fix), f64(temp), f64(tstart), f64(tend)
        atol, rtol, cfactor, sun, hstart = f64(atol), f64(rtol), f64(cfactor), f64(sun), f64(hstart)
        ip = np.ascontiguousarray(ipar, dtype=np.int32)
        rp = np.ascontiguousarray(rpar, dtype=np.float64)
        ist = np.zeros((8, ld), np.int32)
        rst = np.zeros((2, ld), np.float64)
        ierr = np.zeros(ld, np.int32)
        fn = self.lib.kppref_integrate if which == "ref" else self.lib.kppor_integrate
        with quiet_stdout():
            fn(ld, ld, _p(var), _p(fix), _p(temp), _p(cfactor), _p(sun), _p(tstart), _p(tend),
               _p(atol), _p(rtol), _p(ip), _p(rp), _p(hstart), _p(ist), _p(rst), _p(ierr))
        return var, ist, rst, ierr

    def set_sun_ulps(self, u: int):
        """Move SUN by one ulp up (1) / down (-1) at every evaluation (0: off)."""
        self.lib.kppref_set_sun_ulps(ctypes.c_int(int(u)))

    def set_cos_ulps(self, u: int):
        """Move Update_SUN's cos() one ulp up (1) / down (-1) (the `_cs` build)."""
        self.lib.kppref_set_cos_ulps(ctypes.c_int(int(u)))

    def fun_jac(self, var, fix, temp, cfactor, sun, t):
        """Rates, Fun and Jac_SP of one cell (1-D var/fix)."""
        var = np.ascontiguousarray(var, dtype=np.float64)
        fix = np.ascontiguousarray(fix, dtype=np.float64)
        rc = np.zeros(self.nreact)
        vd = np.zeros(self.nvar)
        jv = np.zeros(self.lu_nonzero)
        self.lib.kppref_fun_jac(_p(var), _p(fix), float(temp), float(cfactor),
                                float(-1.0 if sun is None else sun), float(t), _p(rc), _p(vd), _p(jv))
        return rc, vd, jv


def alternates(mech: str, var, fix, temp, tstart, tend, atol, rtol, ipar, rpar, cfactor=None,
               sun=None, hstart=None):
    """VAR after the same integration by the reference under other valid
    last-ulp roundings: compiled with FMA contraction; SUN moved by one ulp up
    and down at every evaluation; Update_SUN's cos() one ulp up and down
    (SUN = (1 + cos)/2 cancels near sunrise and sunset, where a one-ulp
    cosine moves SUN far more than one ulp of SUN does; built for the
    mechanisms that compute SUN from TIME); and pow() of the step-size
    controller one ulp up and down.  Their spread around the reference
    measures how strongly each entry amplifies last-ulp perturbations."""
    out = []
    o3 = OracleLib(mech, "_O3")
    out.append(o3.integrate(var, fix, temp, tstart, tend, atol, rtol, ipar, rpar, cfactor=cfactor,
                            sun=sun, hstart=hstart)[0])
    o = OracleLib(mech)
    for u in (1, -1):
        o.set_sun_ulps(u)
        try:
            out.append(o.integrate(var, fix, temp, tstart, tend, atol, rtol, ipar, rpar,
                                   cfactor=cfactor, sun=sun, hstart=hstart)[0])
        finally:
            o.set_sun_ulps(0)
    # pow() of the step-size controller one ulp up / down (the restatement,
    # bit-identical to the reference with the knob off)
    for u in (1, -1):
        o.lib.kppor_set_pow_ulps(ctypes.c_int(u))
        try:
            out.append(o.integrate(var, fix, temp, tstart, tend, atol, rtol, ipar, rpar,
                                   cfactor=cfactor, sun=sun, hstart=hstart, which="port")[0])
        finally:
            o.lib.kppor_set_pow_ulps(ctypes.c_int(0))
    if lib_path(mech, "_cs").exists():
        cs = OracleLib(mech, "_cs")
        for u in (1, -1):
            cs.set_cos_ulps(u)
            try:
                out.append(cs.integrate(var, fix, temp, tstart, tend, atol, rtol, ipar, rpar,
                                        cfactor=cfactor, sun=sun, hstart=hstart)[0])
            finally:
                cs.set_cos_ulps(0)
    return np.stack(out)


_INTEGRATORS = {"sdirk": ("sdirk", "kppsd"), "rk": ("rk", "kpprk")}


def integrator_lib_path(kind: str, mech: str, opt: str = "") -> Path:
    tag, prefix = _INTEGRATORS[kind]
    return REF_DIR / f"{mech}_{tag}" / f"lib{prefix}_{mech}{opt}.so"


def sdirk_lib_path(mech: str, opt: str = "") -> Path:
    return integrator_lib_path("sdirk", mech, opt)


def rk_lib_path(mech: str, opt: str = "") -> Path:
    return integrator_lib_path("rk", mech, opt)


@contextlib.contextmanager
def quiet_stdout():
    """The reference integrators print a message per failing cell
    (ros_ErrorMsg and its SDIRK / Runge-Kutta counterparts); error-path tests
    make hundreds of thousands of them.  Sends the C library's stdout to
    /dev/null for the length of a call."""
    libc = ctypes.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    try:
        yield
    finally:
        libc.fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(null)


class IntegratorOracle:
    """The reference's own C SDIRK (int/sdirk.c) or Runge-Kutta
    (int/runge_kutta.c) integrator on the mechanism's generated model, per
    cell through oracle/refkpp/batch_driver_sdirk.c / batch_driver_rk.c."""

    kind = "sdirk"

    def __init__(self, mech: str, opt: str = ""):
        self.prefix = _INTEGRATORS[self.kind][1]
        self.lib = ctypes.CDLL(str(integrator_lib_path(self.kind, mech, opt)))
        self._integrate = getattr(self.lib, f"{self.prefix}_integrate")
        self._integrate.argtypes = [ctypes.c_int, ctypes.c_int] + [_vp] * 14
        d = (ctypes.c_int * 5)()
        getattr(self.lib, f"{self.prefix}_dims")(d)
        self.nvar, self.lu_nonzero = d[0], d[4]
        self._sun = getattr(self.lib, f"{self.prefix}_set_sun_ulps")
        self._sun.argtypes = [ctypes.c_int]

    def set_sun_ulps(self, u: int):
        self._sun(u)

    def set_pow_ulps(self, u: int):
        """Moves the integrator's pow() results one ulp (the `_pw` build only)."""
        self.lib.kppref_set_pow_ulps(ctypes.c_int(u))

    def set_cos_ulps(self, u: int):
        """Moves Update_SUN's cos() results one ulp (the `_pw` build only)."""
        self.lib.kppref_set_cos_ulps(ctypes.c_int(u))

    def integrate(self, var, fix, temp, tstart, tend, atol, rtol, icntrl, rcntrl, cfactor=None,
                  sun=None):
        """Returns (var_out, istatus [8][n], rstatus [3][n], ierr): SDIRK's
        ISTATUS[1..8] / RSTATUS[1..3], Runge-Kutta's ISTATUS[0..7] /
        RSTATUS[0..2]."""
        var = np.ascontiguousarray(var, dtype=np.float64).copy()
        n = var.shape[1]
        f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        fix = f64(fix) if fix is not None and np.size(fix) else np.zeros((1, n))
        temp, tstart, tend, atol, rtol = f64(temp), f64(tstart), f64(tend), f64(atol), f64(rtol)
        cfactor, sun = f64(cfactor), f64(sun)
        ic = np.ascontiguousarray(icntrl, dtype=np.int32)
        rc = np.ascontiguousarray(rcntrl, dtype=np.float64)
        ist = np.zeros((8, n), np.int32)
        rst = np.zeros((3, n))
        ierr = np.zeros(n, np.int32)
        with quiet_stdout():
            self._integrate(n, n, _p(var), _p(fix), _p(temp), _p(cfactor), _p(sun),
                            _p(tstart), _p(tend), _p(atol), _p(rtol), _p(ic), _p(rc), _p(ist),
                            _p(rst), _p(ierr))
        return var, ist, rst, ierr


class SdirkOracle(IntegratorOracle):
    kind = "sdirk"


class RkOracle(IntegratorOracle):
    kind = "rk"

    def decomp_cmplx(self, jr, ji):
        """The reference's KppDecompCmplxR (util/sutil.c:28-59) in place."""
        return int(self.lib.kpprk_decomp_cmplx(_p(jr), _p(ji)))

    def solve_cmplx(self, jr, ji, xr, xi):
        """The reference's KppSolveCmplxR (util/sutil.c:64-87) in place."""
        self.lib.kpprk_solve_cmplx(_p(jr), _p(ji), _p(xr), _p(xi))


def adj_lib_path(mech: str, opt: str = "") -> Path:
    return REF_DIR / f"{mech}_adj" / f"libkppadj_{mech}{opt}.so"


class AdjOracle:
    """The reference's own C RosenbrockADJ (int/rosenbrock_adj.c) on the
    mechanism's generated model with its Hessian, per cell through
    oracle/refkpp/batch_driver_adj.c."""

    def __init__(self, mech: str, opt: str = ""):
        self.lib = ctypes.CDLL(str(adj_lib_path(mech, opt)))
        self._integrate = self.lib.kppadj_integrate
        self._integrate.argtypes = ([ctypes.c_int, ctypes.c_int] + [_vp] * 9 + [ctypes.c_int]
                                    + [_vp] * 3 + [ctypes.c_int] + [_vp] * 3)
        d = (ctypes.c_int * 5)()
        self.lib.kppadj_dims(d)
        self.nvar = d[0]

    def integrate(self, var, fix, temp, tstart, tend, atol, rtol, lam, icntrl, rcntrl, bufsize,
                  cfactor=None, sun=None):
        """Returns (var_out, lam_out, istatus [8][n], rstatus [3][n], ierr):
        ISTATUS[1..8], RSTATUS[1..3]; lam [NADJ * NVAR][n]."""
        var = np.ascontiguousarray(var, dtype=np.float64).copy()
        lam = np.ascontiguousarray(lam, dtype=np.float64).copy()
        n = var.shape[1]
        nadj = lam.shape[0] // self.nvar
        f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        fix = f64(fix) if fix is not None and np.size(fix) else np.zeros((1, n))
        temp, tstart, tend, atol, rtol = f64(temp), f64(tstart), f64(tend), f64(atol), f64(rtol)
        cfactor, sun = f64(cfactor), f64(sun)
        ic = np.ascontiguousarray(icntrl, dtype=np.int32)
        rc = np.ascontiguousarray(rcntrl, dtype=np.float64)
        ist = np.zeros((8, n), np.int32)
        rst = np.zeros((3, n))
        ierr = np.zeros(n, np.int32)
        with quiet_stdout():
            self._integrate(n, n, _p(var), _p(fix), _p(temp), _p(cfactor), _p(sun), _p(tstart),
                            _p(tend), _p(atol), _p(rtol), nadj, _p(lam), _p(ic), _p(rc),
                            int(bufsize), _p(ist), _p(rst), _p(ierr))
        return var, lam, ist, rst, ierr


def integrator_alternates(kind: str, mech: str, var, fix, temp, tstart, tend, atol, rtol,
                          icntrl, rcntrl, cfactor=None, sun=None):
    """VAR after the same SDIRK or Runge-Kutta integration by the reference
    under other valid last-ulp roundings: compiled with FMA contraction; SUN
    one ulp up and down at every evaluation; the integrator's pow() one ulp
    up and down, and one ulp off in a direction that varies from call to call
    (two hashes of the arguments: the step-size factor, the LU reuse test and
    the Newton convergence tests decide on pow results, so per-call errors
    can change the step sequence); Update_SUN's cos() one ulp up and down (SUN = (1 + cos)/2 cancels
    near sunrise and sunset, where a one-ulp cosine moves SUN far more than
    one ulp of SUN does)."""
    cls = SdirkOracle if kind == "sdirk" else RkOracle
    args = (var, fix, temp, tstart, tend, atol, rtol, icntrl, rcntrl)
    out = [cls(mech, "_O3").integrate(*args, cfactor=cfactor, sun=sun)[0]]
    o = cls(mech)
    for u in (1, -1):
        o.set_sun_ulps(u)
        try:
            out.append(o.integrate(*args, cfactor=cfactor, sun=sun)[0])
        finally:
            o.set_sun_ulps(0)
    pw = cls(mech, "_pw")
    for knob, values in ((pw.set_pow_ulps, (1, -1, 2, 3)), (pw.set_cos_ulps, (1, -1))):
        for u in values:
            knob(u)
            try:
                out.append(pw.integrate(*args, cfactor=cfactor, sun=sun)[0])
            finally:
                knob(0)
    return np.stack(out)


def sdirk_alternates(mech: str, *args, **kw):
    return integrator_alternates("sdirk", mech, *args, **kw)


def rk_alternates(mech: str, *args, **kw):
    return integrator_alternates("rk", mech, *args, **kw)
