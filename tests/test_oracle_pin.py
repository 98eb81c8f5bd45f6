"""The oracle, pinned (CPU).

  * the documented small_strato species order and LU pattern
    (docs/source/output/code_f90.rst:234-241, 500-505) against the reference
    generator built here;
  * the CPU restatement oracle/ros_oracle.c against the reference's own
    Rosenbrock (int/rosenbrock.c, run through oracle/refkpp/batch_driver.c):
    bit-identical results, statistics and error codes on seeded batches,
    including every error path;
  * the restatement against the committed golden vectors.
"""
import json

import numpy as np
import pytest

from kpp_b200 import make_controls, workloads
from oracle_lib import OracleLib, ensure_built

MECHS = ["small_strato", "saprc99", "mcm_isoprene"]

pytestmark = pytest.mark.skipif(not ensure_built(), reason="oracle libraries not built")


class _View:
    def __init__(self, o):
        self.o, self.nvar, self.species = o, o.nvar, o.species

    def initial_values(self):
        c, cf = self.o.initial_values()
        return list(c), cf


def test_small_strato_matches_documented_structure():
    o = OracleLib("small_strato")
    assert o.species == ["O1D", "O", "O3", "NO", "NO2", "M", "O2"]
    irow, icol, crow, diag = o.lu_pattern()
    # docs/source/output/code_f90.rst:500-505 (1-based there)
    assert (icol + 1).tolist() == [1, 3, 1, 2, 3, 5, 1, 2, 3, 4, 5, 2, 3, 4, 5, 2, 3, 4, 5]
    assert (irow + 1).tolist() == [1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5]
    assert (crow + 1).tolist() == [1, 3, 7, 12, 16, 20]
    assert (diag + 1).tolist() == [1, 4, 9, 14, 19, 20]


@pytest.mark.parametrize("mech", MECHS)
def test_structure_matches_golden(mech, golden_dir):
    o = OracleLib(mech)
    g = json.loads((golden_dir / f"structure_{mech}.json").read_text())
    irow, icol, crow, diag = o.lu_pattern()
    assert o.species == g["species"]
    # fixed species: NSPEC - NVAR (the C model pads NFIX to 1 when there are none)
    assert [o.nvar, o.nspec - o.nvar, o.nreact, o.lu_nonzero] == [g["nvar"], g["nfix"], g["nreact"],
                                                                 g["lu_nonzero"]]
    assert icol.tolist() == g["lu_icol"] and crow.tolist() == g["lu_crow"]
    assert diag.tolist() == g["lu_diag"] and irow.tolist() == g["lu_irow"]


def _both(o, wl, ipar, rpar, atol=None, rtol=None, k=0):
    t0, t1 = wl.step_bounds(k)
    atol = wl.atol if atol is None else atol
    rtol = wl.rtol if rtol is None else rtol
    a = o.integrate(wl.var, wl.fix, wl.temp, t0, t1, atol, rtol, ipar, rpar,
                    cfactor=wl.cfactor, sun=wl.sun, which="ref")
    b = o.integrate(wl.var, wl.fix, wl.temp, t0, t1, atol, rtol, ipar, rpar,
                    cfactor=wl.cfactor, sun=wl.sun, which="port")
    return a, b


def _assert_identical(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("method", ["ros2", "ros3", "ros4", "rodas3", "rodas4"])
@pytest.mark.parametrize("mech,n", [("small_strato", 96), ("saprc99", 16), ("mcm_isoprene", 3)])
def test_restatement_bit_identical_to_reference(mech, n, method):
    o = OracleLib(mech)
    wl = workloads.for_mechanism(_View(o), mech, n, seed=123)
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    a, b = _both(o, wl, ipar, rpar)
    _assert_identical(a, b)
    assert (a[3] == 1).all()


@pytest.mark.parametrize("ctl,tol,code", [
    (dict(method=0), {}, -2), (dict(method=6), {}, -2), (dict(method=7), {}, -2),
    (dict(max_steps=-3), {}, -1), (dict(hmin=-1.0), {}, -3), (dict(hmax=-1.0), {}, -3),
    (dict(hstart=-1.0), {}, -3), (dict(facmin=-1.0), {}, -4), (dict(facmax=-1.0), {}, -4),
    (dict(facrej=-1.0), {}, -4), (dict(facsafe=-1.0), {}, -4), ({}, {"rtol": 1e-16}, -5),
    ({}, {"rtol": 1.5}, -5), ({}, {"atol": -1.0}, -5), (dict(max_steps=1), {}, -6),
    (dict(hmax=1e-300), {}, -7),
])
def test_restatement_error_paths_identical(ctl, tol, code):
    o = OracleLib("small_strato")
    wl = workloads.for_mechanism(_View(o), "small_strato", 8, seed=5)
    ipar, rpar = make_controls(scalar_tol=True, **{"method": "rodas3", **ctl})
    atol = np.array([tol.get("atol", 1.0)])
    rtol = np.array([tol.get("rtol", 1e-3)])
    a, b = _both(o, wl, ipar, rpar, atol, rtol)
    _assert_identical(a, b)
    assert (a[3] == code).all()


def test_restatement_vector_tolerances_and_warm_start():
    o = OracleLib("small_strato")
    wl = workloads.for_mechanism(_View(o), "small_strato", 32, seed=9)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=False)
    atol = np.linspace(0.5, 2.0, o.nvar)
    rtol = np.linspace(1e-4, 1e-3, o.nvar)
    t0, t1 = wl.step_bounds(0)
    hs = np.full(32, 30.0)
    a = o.integrate(wl.var, wl.fix, wl.temp, t0, t1, atol, rtol, ipar, rpar, hstart=hs, which="ref")
    b = o.integrate(wl.var, wl.fix, wl.temp, t0, t1, atol, rtol, ipar, rpar, hstart=hs, which="port")
    _assert_identical(a, b)


@pytest.mark.parametrize("mech", MECHS)
def test_restatement_reproduces_golden_vectors(mech, golden_dir):
    g = np.load(golden_dir / f"integrate_{mech}.npz")
    o = OracleLib(mech)
    var = g["var0"].copy()
    hs = np.zeros(var.shape[1])
    cf = g["cfactor"] if g["cfactor"].size else None
    sun = g["sun"] if g["sun"].size else None
    for k in range(g["var"].shape[0]):
        t0 = g["tstart"] + k * float(g["dt"])
        var, ist, rst, ierr = o.integrate(var, g["fix"], g["temp"], t0, t0 + float(g["dt"]),
                                          g["atol"], g["rtol"], g["ipar"], g["rpar"], cfactor=cf,
                                          sun=sun, hstart=hs, which="port")
        hs = rst[1].copy()
        np.testing.assert_array_equal(var, g["var"][k])
        np.testing.assert_array_equal(ist, g["istatus"][k])
        np.testing.assert_array_equal(ierr, g["ierr"][k])


@pytest.mark.parametrize("mech", ["small_strato", "saprc99"])
def test_rounding_alternate_builds_reproduce_reference_with_knobs_off(mech):
    """The builds behind the parity bar's rounding alternates (the reference
    with Update_SUN's cos(), or the SDIRK integrator's pow() and cos(),
    routed through a one-ulp knob) are the reference itself with the knob
    off, and move results with it on."""
    from oracle_lib import SdirkOracle, lib_path, sdirk_lib_path
    if not (lib_path(mech, "_cs").exists() and sdirk_lib_path(mech, "_pw").exists()):
        pytest.skip("rounding-alternate builds not present")
    o = OracleLib(mech)
    n = 64
    wl = workloads.for_mechanism(_View(o), mech, n, seed=17)
    fix = wl.fix if wl.fix.shape[0] else np.zeros((1, n))
    # a window across sunrise or sunset, where the cosine matters
    t0, t1 = wl.step_bounds(3)
    kw = dict(cfactor=wl.cfactor, sun=None)  # SUN from TIME: Update_SUN runs
    cs = OracleLib(mech, "_cs")
    ref = o.integrate(wl.var, fix, wl.temp, t0, t1, wl.atol, wl.rtol, wl.ipar, wl.rpar, **kw)
    got = cs.integrate(wl.var, fix, wl.temp, t0, t1, wl.atol, wl.rtol, wl.ipar, wl.rpar, **kw)
    for a, b in zip(ref, got):
        np.testing.assert_array_equal(a, b)
    cs.set_cos_ulps(1)
    try:
        moved = cs.integrate(wl.var, fix, wl.temp, t0, t1, wl.atol, wl.rtol, wl.ipar, wl.rpar, **kw)
    finally:
        cs.set_cos_ulps(0)
    assert not np.array_equal(moved[0], ref[0])

    ic, rc = [0] * 20, [0.0] * 20
    ic[1], ic[2] = 1, 3
    sd, pw = SdirkOracle(mech), SdirkOracle(mech, "_pw")
    ref = sd.integrate(wl.var, fix, wl.temp, t0, t1, wl.atol, wl.rtol, ic, rc, **kw)
    got = pw.integrate(wl.var, fix, wl.temp, t0, t1, wl.atol, wl.rtol, ic, rc, **kw)
    for a, b in zip(ref, got):
        np.testing.assert_array_equal(a, b)
    for knob in (pw.set_pow_ulps, pw.set_cos_ulps):
        knob(-1)
        try:
            moved = pw.integrate(wl.var, fix, wl.temp, t0, t1, wl.atol, wl.rtol, ic, rc, **kw)
        finally:
            knob(0)
        assert not np.array_equal(moved[0], ref[0])
