"""The warp-per-cell kernel (kpp_b200/csrc/kpp_coop.cuh) against the
thread-per-cell kernel, which the parity tests pin to the reference (GPU).

Both perform the same operations in the same order, so every output must be
identical bit for bit: VAR, ISTATUS, RSTATUS and IERR, for every Rosenbrock
method, every control and error path, scalar and vector tolerances,
autonomous and time-dependent calls, single calls with any starting step,
chained calls in any queue order, ragged batches and a leading dimension
larger than the batch.  The kernel runs launches whose rate constants are
fixed for the call (SUN given per cell); small_strato is run that way too.
"""
import numpy as np
import pytest
import torch

from kpp_b200 import load, make_controls, workloads

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(
        device="cuda", dtype=dtype)


def _sun(wl, n):
    """Per-cell SUN: the workload's own, or for small_strato Update_SUN's value
    at each cell's start time (the rates are then fixed over the call)."""
    if wl.sun is not None:
        return wl.sun
    rng = np.random.default_rng(9)
    return np.where(rng.uniform(size=n) < 0.3, 0.0, rng.uniform(0.0, 1.0, n))


def _run(m, which, fn):
    m.set_kernel(which)
    try:
        assert m.kernel() == which
        out = fn()
        torch.cuda.synchronize()
        return [x.cpu().numpy() for x in out]
    finally:
        m.set_kernel("auto")


def _single(m, wl, ipar, rpar, n, ld=None, hstart=None, atol=None, rtol=None):
    ld = ld or n
    pad = lambda a: None if a is None else np.concatenate(
        [a, np.zeros(a.shape[:-1] + (ld - a.shape[-1],))], axis=-1) if ld > a.shape[-1] else a
    t0, t1 = wl.step_bounds(0)
    sun = _sun(wl, n)

    def fn():
        var = dev(pad(wl.var))
        r = m.rosenbrock(var, dev(pad(wl.fix)), dev(pad(wl.temp)), dev(pad(t0)), dev(pad(t1)),
                         dev(wl.atol if atol is None else atol),
                         dev(wl.rtol if rtol is None else rtol), ipar, rpar,
                         cfactor=dev(pad(wl.cfactor)), sun=dev(pad(sun)),
                         hstart=dev(pad(hstart)), ncells=n)
        return var, r.istatus, r.rstatus, r.ierr
    return fn


def _same(a, b):
    for x, y, nm in zip(a, b, ("var", "istatus", "rstatus", "ierr")):
        np.testing.assert_array_equal(x, y, err_msg=nm)


@pytest.mark.parametrize("method", ["ros2", "ros3", "ros4", "rodas3", "rodas4"])
@pytest.mark.parametrize("autonomous", [False, True])
def test_every_method_bit_identical(method, autonomous):
    m = load("saprc99")
    n = 500
    wl = workloads.for_mechanism(m, "saprc99_uniform95", n, seed=41)
    ipar, rpar = make_controls(method=method, scalar_tol=True, autonomous=autonomous)
    hs = np.where(np.arange(n) % 3 == 0, 0.0, np.geomspace(1e-6, 100.0, n))
    fn = _single(m, wl, ipar, rpar, n, hstart=hs)
    _same(_run(m, "thread", fn), _run(m, "warp", fn))


def _controls_cases():
    base = dict(method="rodas3", scalar_tol=True)
    return [
        ("bad_method", dict(base, method=0), {}),
        ("bad_method_7", dict(base, method=7), {}),
        ("neg_max_steps", dict(base, max_steps=-1), {}),
        ("neg_hmin", dict(base, hmin=-1.0), {}),
        ("neg_facrej", dict(base, facrej=-0.5), {}),
        ("tiny_rtol", dict(base), {"rtol": 1e-17}),
        ("zero_atol", dict(base), {"atol": 0.0}),
        ("max_steps_3", dict(base, max_steps=3), {}),
        ("tiny_hmax", dict(base, hmax=1e-300), {}),
        ("hmin_large", dict(base, hmin=50.0), {}),
        ("facmax_facsafe", dict(base, facmax=2.0, facsafe=0.5, facrej=0.3), {}),
        ("vector_tol", dict(method="rodas4", scalar_tol=False), {"vector": True}),
        ("backward", dict(base), {"backward": True}),
    ]


@pytest.mark.parametrize("name,ctl,tol", _controls_cases(), ids=[c[0] for c in _controls_cases()])
def test_controls_and_error_paths_bit_identical(name, ctl, tol):
    m = load("saprc99")
    n = 200
    wl = workloads.for_mechanism(m, "saprc99_uniform95", n, seed=43)
    ipar, rpar = make_controls(**ctl)
    atol = rtol = None
    if tol.get("vector"):
        atol = np.linspace(1e-3, 1e-1, m.nvar)
        rtol = np.linspace(1e-4, 1e-3, m.nvar)
    elif "atol" in tol or "rtol" in tol:
        atol = np.array([tol.get("atol", 1e-2)])
        rtol = np.array([tol.get("rtol", 1e-3)])
    if tol.get("backward"):
        t0, t1 = wl.step_bounds(0)
        wl.tstart = t1.copy()
        wl.dt = -wl.dt
    fn = _single(m, wl, ipar, rpar, n, atol=atol, rtol=rtol)
    a, b = _run(m, "thread", fn), _run(m, "warp", fn)
    _same(a, b)
    if name.startswith(("bad", "neg", "tiny_rtol", "zero")):
        assert (a[3] < 0).all()


def test_ragged_batch_and_larger_leading_dimension():
    m = load("saprc99")
    n = 3001  # not a multiple of a CTA's warps
    wl = workloads.for_mechanism(m, "saprc99_classes", n, seed=44)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    fn = _single(m, wl, ipar, rpar, n, ld=n + 37)
    a, b = _run(m, "thread", fn), _run(m, "warp", fn)
    _same(a, b)
    # the padding columns are untouched
    assert (b[0][:, n:] == 0).all()


def test_small_strato_with_per_cell_sun():
    m = load("small_strato")
    n = 777
    wl = workloads.for_mechanism(m, "small_strato", n, seed=45)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    fn = _single(m, wl, ipar, rpar, n)
    _same(_run(m, "thread", fn), _run(m, "warp", fn))


@pytest.mark.parametrize("ordered", [False, True])
def test_chained_calls_in_queue_order_bit_identical(ordered):
    m = load("saprc99")
    n, ncalls = 900, 4
    wl = workloads.for_mechanism(m, "saprc99_classes", n, seed=46)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    order = np.random.default_rng(3).permutation(n).astype(np.int32) if ordered else None

    def fn():
        var = dev(wl.var)
        r = m.rosenbrock_chain(var, dev(wl.fix), dev(wl.temp), dev(wl.tstart), wl.dt, ncalls,
                               dev(wl.atol), dev(wl.rtol), ipar, rpar, cfactor=dev(wl.cfactor),
                               sun=dev(wl.sun),
                               order=None if order is None else dev(order, torch.int32))
        return var, r.istatus, r.rstatus, r.ierr
    _same(_run(m, "thread", fn), _run(m, "warp", fn))


def test_update_sun_launches_fall_back_to_the_thread_kernel():
    """Rates that follow Update_SUN(TIME) are not fixed for the call: the
    launch runs on the thread-per-cell kernel whatever the choice."""
    m = load("small_strato")
    n = 100
    wl = workloads.for_mechanism(m, "small_strato", n, seed=47)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    t0, t1 = wl.step_bounds(0)

    def fn():
        var = dev(wl.var)
        r = m.rosenbrock(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol),
                         dev(wl.rtol), ipar, rpar)
        return var, r.istatus, r.rstatus, r.ierr
    _same(_run(m, "thread", fn), _run(m, "warp", fn))
