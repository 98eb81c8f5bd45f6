"""The mechanism library built on KPP's own generator (#LANGUAGE CUDA) against
the one built on kppcu (GPU).

libkpp_b200_<mech>_kpproute.so runs the same kernels as libkpp_b200_<mech>.so
with the rate constants, Fun, Jac_SP, KppDecomp and KppSolve that KPP's
generator writes with the CUDA target (kpp_b200/kppgen).  Both routes emit the
C target's arithmetic operation for operation (tests/test_kpp_route.py checks
that on the host), so every integrator output must be identical bit for bit:
VAR, ISTATUS, RSTATUS and IERR, on every Rosenbrock method, the SDIRK and the
Runge-Kutta integrators, fixed and Update_SUN rates; and the building blocks
(fun_jac, decomp_solve) give the same arrays.  The kppcu library runs its
thread-per-cell kernel, the one the generator-route library has.
"""
import numpy as np
import pytest
import torch

from kpp_b200 import Mechanism, build, load, make_controls, workloads

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(
        device="cuda", dtype=dtype)


def pair(mech):
    path = build.library_path(mech, "kpp")
    if not path.exists():
        pytest.skip(f"{path.name} not built (KPP's sources were not found at build time)")
    return load(mech), Mechanism(mech, path=path)


def _host(*ts):
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in ts]


def _same(a, b, what):
    for x, y, nm in zip(a, b, ("var", "istatus", "rstatus", "ierr")):
        np.testing.assert_array_equal(x, y, err_msg=f"{what}: {nm}")


def _rosenbrock(m, wl, ipar, rpar, t0, t1, sun):
    var = dev(wl.var)
    r = m.rosenbrock(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol),
                     dev(wl.rtol), ipar, rpar, cfactor=dev(wl.cfactor), sun=dev(sun))
    return _host(var, r.istatus, r.rstatus, r.ierr)


def _with_thread_kernel(m, fn):
    m.set_kernel("thread")
    try:
        return fn()
    finally:
        m.set_kernel("auto")


@pytest.mark.parametrize("method", ["ros2", "ros3", "ros4", "rodas3", "rodas4"])
def test_rosenbrock_saprc99_bit_identical(method):
    kppcu, route = pair("saprc99")
    assert route.kernel() == "thread"
    n = 512
    wl = workloads.for_mechanism(kppcu, "saprc99_uniform95", n, seed=51)
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    t0, t1 = wl.step_bounds(0)
    a = _with_thread_kernel(kppcu, lambda: _rosenbrock(kppcu, wl, ipar, rpar, t0, t1, wl.sun))
    b = _rosenbrock(route, wl, ipar, rpar, t0, t1, wl.sun)
    assert (a[3] == 1).all()
    _same(a, b, method)


@pytest.mark.parametrize("step", [0, 5])
def test_rosenbrock_small_strato_update_sun_bit_identical(step):
    """SUN from Update_SUN(TIME) inside the integrator: the rates are
    recomputed at every stage time."""
    kppcu, route = pair("small_strato")
    n = 1024
    wl = workloads.for_mechanism(kppcu, "small_strato", n, seed=52)
    ipar, rpar = make_controls(method="rodas4", scalar_tol=True)
    t0, t1 = wl.step_bounds(step)
    a = _with_thread_kernel(kppcu, lambda: _rosenbrock(kppcu, wl, ipar, rpar, t0, t1, None))
    b = _rosenbrock(route, wl, ipar, rpar, t0, t1, None)
    _same(a, b, f"step {step}")


def test_rosenbrock_chain_saprc99_bit_identical():
    kppcu, route = pair("saprc99")
    n, ncalls = 700, 3
    wl = workloads.for_mechanism(kppcu, "saprc99_classes", n, seed=53)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)

    def run(m):
        var = dev(wl.var)
        r = m.rosenbrock_chain(var, dev(wl.fix), dev(wl.temp), dev(wl.tstart), wl.dt, ncalls,
                               dev(wl.atol), dev(wl.rtol), ipar, rpar, cfactor=dev(wl.cfactor),
                               sun=dev(wl.sun))
        return _host(var, r.istatus, r.rstatus, r.ierr)
    _same(_with_thread_kernel(kppcu, lambda: run(kppcu)), run(route), "chain")


def _other(m, wl, which, ic, rc):
    t0, t1 = wl.step_bounds(0)
    var = dev(wl.var)
    f = m.sdirk if which == "sdirk" else m.runge_kutta
    r = f(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol), dev(wl.rtol), ic, rc,
          cfactor=dev(wl.cfactor), sun=dev(wl.sun))
    return _host(var, r.istatus, r.rstatus, r.ierr)


@pytest.mark.parametrize("mech,which,method", [("small_strato", "sdirk", 3),
                                               ("saprc99", "sdirk", 1),
                                               ("small_strato", "rk", 0),
                                               ("saprc99", "rk", 2)])
def test_sdirk_and_runge_kutta_bit_identical(mech, which, method):
    kppcu, route = pair(mech)
    n = 256
    wl = workloads.for_mechanism(kppcu, mech, n, seed=54)
    ic, rc = [0] * 20, [0.0] * 20
    ic[1] = 1 if wl.atol.size == 1 else 0
    # ICNTRL[2]: the SDIRK method (int/sdirk.c) or the Runge-Kutta family
    # member (int/runge_kutta.c)
    ic[2] = method
    _same(_other(kppcu, wl, which, ic, rc), _other(route, wl, which, ic, rc), f"{which} {method}")


@pytest.mark.parametrize("mech", ["small_strato", "saprc99"])
def test_building_blocks_identical(mech):
    kppcu, route = pair(mech)
    n = 333
    wl = workloads.for_mechanism(kppcu, mech, n, seed=55)
    t0, _ = wl.step_bounds(0)
    sun = wl.sun if wl.sun is not None else np.full(n, 0.7)
    out = []
    for m in (kppcu, route):
        rc, vd, jv = m.fun_jac(dev(wl.var), dev(wl.fix), dev(wl.temp), float(t0[0]),
                               cfactor=dev(wl.cfactor), sun=dev(sun))
        lu = -jv.clone()
        lu[torch.as_tensor(m.lu_pattern()[3][:-1], device="cuda", dtype=torch.long)] += 1.0 / 60.0
        x = dev(np.random.default_rng(5).standard_normal((m.nvar, n)))
        ising = m.decomp_solve(lu, x)
        out.append(_host(vd, jv, lu, x, ising))
    for a, b, nm in zip(out[0], out[1], ("vdot", "jvs", "lu", "x", "ising")):
        np.testing.assert_array_equal(a, b, err_msg=nm)
