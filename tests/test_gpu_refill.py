"""The lane-granular work queue of kpp_b200_rosenbrock_chain (GPU).

With kpp_b200_set_queue_lanes(1) each lane takes its own next cell and the
lanes' cells advance one step attempt at a time together, however far apart
they are (integrate_refill in kpp_b200/csrc/kpp_rosenbrock.cu).  Every cell
performs the operations of the warp-granular queue in the same order, which
tests/test_gpu_chain.py ties to chained kpp_b200_rosenbrock launches, so all
outputs must be identical bit for bit: VAR, ISTATUS, RSTATUS and IERR, for
every method, chained calls, any queue order, per-cell starting steps (some
of them invalid), the control and error paths, Update_SUN rates, backward
integration and vector tolerances.  Both runs use the thread-per-cell kernel.
"""
import numpy as np
import pytest
import torch

from kpp_b200 import load, make_controls, workloads

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(
        device="cuda", dtype=dtype)


def run_both(m, wl, ipar, rpar, ncalls, order=None, hstart=None, dt=None, atol=None, rtol=None):
    out = []
    for lanes in (False, True):
        m.set_kernel("thread")
        m.set_queue_lanes(lanes)
        try:
            assert m.queue_lanes() == lanes
            var = dev(wl.var)
            r = m.rosenbrock_chain(var, dev(wl.fix), dev(wl.temp), dev(wl.tstart),
                                   wl.dt if dt is None else dt, ncalls,
                                   dev(wl.atol if atol is None else atol),
                                   dev(wl.rtol if rtol is None else rtol), ipar, rpar,
                                   cfactor=dev(wl.cfactor), sun=dev(wl.sun),
                                   hstart=dev(hstart), order=dev(order, torch.int32))
            torch.cuda.synchronize()
            out.append([x.cpu().numpy() for x in (var, r.istatus, r.rstatus, r.ierr)])
        finally:
            m.set_queue_lanes(True)  # the default
            m.set_kernel("auto")
    for x, y, nm in zip(out[0], out[1], ("var", "istatus", "rstatus", "ierr")):
        np.testing.assert_array_equal(x, y, err_msg=nm)
    return out[1]


@pytest.mark.parametrize("method", ["ros2", "ros3", "ros4", "rodas3", "rodas4"])
def test_every_method_bit_identical(method):
    m = load("saprc99")
    n = 3001
    wl = workloads.for_mechanism(m, "saprc99_classes", n, seed=61)
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    order = np.random.default_rng(7).permutation(n).astype(np.int32)
    hs = np.where(np.arange(n) % 4 == 0, 0.0, np.geomspace(1e-7, 30.0, n))
    var, ist, rst, ierr = run_both(m, wl, ipar, rpar, 2, order=order, hstart=hs)
    assert (ierr == 1).all()


def test_per_cell_errors_and_step_limits():
    """Cells whose Hstart is negative fail validation (-3) while their
    neighbours integrate; a step limit ends other cells' calls with -6 in
    mid-queue; every lane then goes on with its next call or cell."""
    m = load("saprc99")
    n = 1500
    wl = workloads.for_mechanism(m, "saprc99_uniform95", n, seed=62)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True, max_steps=30)
    hs = np.where(np.arange(n) % 7 == 3, -1.0, 0.0)
    _, _, _, ierr = run_both(m, wl, ipar, rpar, 3, hstart=hs)
    assert (ierr[np.arange(n) % 7 == 3] == -3).all()
    assert (ierr == -6).any() and (ierr == 1).any()


@pytest.mark.parametrize("case", ["bad_method", "neg_facrej", "tiny_rtol", "tiny_hmax",
                                  "hmin_large", "vector_tol", "backward"])
def test_controls_and_error_paths_bit_identical(case):
    m = load("saprc99")
    n = 700
    wl = workloads.for_mechanism(m, "saprc99_classes", n, seed=63)
    ctl = dict(method="rodas3", scalar_tol=True)
    atol = rtol = None
    dt = None
    if case == "bad_method":
        ctl["method"] = 7
    elif case == "neg_facrej":
        ctl["facrej"] = -0.5
    elif case == "tiny_rtol":
        rtol = np.array([1e-17])
    elif case == "tiny_hmax":
        ctl["hmax"] = 1e-300
    elif case == "hmin_large":
        ctl["hmin"] = 50.0
    elif case == "vector_tol":
        ctl = dict(method="rodas4", scalar_tol=False)
        atol = np.linspace(1e-3, 1e-1, m.nvar)
        rtol = np.linspace(1e-4, 1e-3, m.nvar)
    elif case == "backward":
        dt = -wl.dt
    ipar, rpar = make_controls(**ctl)
    _, _, _, ierr = run_both(m, wl, ipar, rpar, 2, dt=dt, atol=atol, rtol=rtol)
    if case in ("bad_method", "neg_facrej", "tiny_rtol"):
        assert (ierr < 0).all()


def test_small_strato_update_sun_chained():
    m = load("small_strato")
    n = 2048
    wl = workloads.for_mechanism(m, "small_strato", n, seed=64)
    ipar, rpar = make_controls(method="rodas4", scalar_tol=True)
    _, _, _, ierr = run_both(m, wl, ipar, rpar, 4)
    assert (ierr == 1).all()


def test_fewer_cells_than_lanes_and_empty_batch():
    m = load("saprc99")
    wl = workloads.for_mechanism(m, "saprc99_uniform95", 37, seed=65)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    run_both(m, wl, ipar, rpar, 1)
    m.set_kernel("thread")
    m.set_queue_lanes(True)
    try:
        z = torch.zeros(m.nvar, 0, dtype=torch.float64, device="cuda")
        e = torch.zeros(0, dtype=torch.float64, device="cuda")
        r = m.rosenbrock_chain(z, torch.zeros(m.nfix, 0, dtype=torch.float64, device="cuda"), e,
                               e, 600.0, 1, dev(wl.atol), dev(wl.rtol), ipar, rpar)
        torch.cuda.synchronize()
        assert r.ierr.numel() == 0
    finally:
        m.set_queue_lanes(True)  # the default
        m.set_kernel("auto")
