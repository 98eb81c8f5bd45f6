"""kpp_b200_rosenbrock_chain (the driver loop over INTEGRATE in one persistent
work-queue launch) against chained single calls of kpp_b200_rosenbrock, which
the parity tests pin to the reference: equal bit for bit, for any queue order.
"""
import numpy as np
import pytest
import torch

from kpp_b200 import load, make_controls, workloads

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def sequential_calls(m, wl, ncalls, ipar, rpar, hstart=None):
    """ncalls kpp_b200_rosenbrock launches chained as INTEGRATE's callers do."""
    var = dev(wl.var)
    fix, temp, atol, rtol = dev(wl.fix), dev(wl.temp), dev(wl.atol), dev(wl.rtol)
    cf = dev(wl.cfactor) if wl.cfactor is not None else None
    sun = dev(wl.sun) if wl.sun is not None else None
    t0 = dev(wl.tstart)
    hs = hstart
    ist_sum, ierr_first = None, None
    for k in range(ncalls):
        t1 = t0 + wl.dt
        r = m.rosenbrock(var, fix, temp, t0, t1, atol, rtol, ipar, rpar, cfactor=cf, sun=sun,
                         hstart=hs)
        ist_sum = r.istatus.clone() if k == 0 else ist_sum + r.istatus
        ierr_first = r.ierr.clone() if k == 0 else torch.where(ierr_first == 1, r.ierr,
                                                                ierr_first)
        hs = r.rstatus[1].clone()
        t0 = t1
    torch.cuda.synchronize()
    return var, ist_sum, r.rstatus, ierr_first


def chained(m, wl, ncalls, ipar, rpar, hstart=None, order=None):
    var = dev(wl.var)
    cf = dev(wl.cfactor) if wl.cfactor is not None else None
    sun = dev(wl.sun) if wl.sun is not None else None
    r = m.rosenbrock_chain(var, dev(wl.fix), dev(wl.temp), dev(wl.tstart), wl.dt, ncalls,
                           dev(wl.atol), dev(wl.rtol), ipar, rpar, cfactor=cf, sun=sun,
                           hstart=hstart, order=order)
    torch.cuda.synchronize()
    return var, r.istatus, r.rstatus, r.ierr


def assert_same(a, b):
    for x, y, nm in zip(a, b, ("var", "istatus", "rstatus", "ierr")):
        np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy(), err_msg=nm)


@pytest.mark.parametrize("mech,wname,ncells,ncalls", [
    ("small_strato", "small_strato", 1000, 6),
    ("saprc99", "saprc99_classes", 700, 3),
])
def test_chain_equals_chained_single_calls(mech, wname, ncells, ncalls):
    m = load(mech)
    wl = workloads.for_mechanism(m, wname, ncells, seed=5)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    assert_same(chained(m, wl, ncalls, ipar, rpar), sequential_calls(m, wl, ncalls, ipar, rpar))


def test_chain_any_queue_order_and_hstart():
    m = load("saprc99")
    n = 900
    wl = workloads.for_mechanism(m, "saprc99_uniform95", n, seed=6)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    hs = dev(10.0 ** np.random.default_rng(1).uniform(-6, 1, n))
    ref = sequential_calls(m, wl, 2, ipar, rpar, hstart=hs)
    perm = dev(np.random.default_rng(2).permutation(n).astype(np.int32), torch.int32)
    rev = dev(np.arange(n - 1, -1, -1, dtype=np.int32), torch.int32)
    for order in (None, perm, rev):
        assert_same(chained(m, wl, 2, ipar, rpar, hstart=hs, order=order), ref)


def test_chain_keeps_first_failure():
    """A step limit that some calls exceed: IERR of the first failing call is
    kept (-6), later calls still run, counters are summed."""
    m = load("saprc99")
    wl = workloads.for_mechanism(m, "saprc99_uniform95", 512, seed=7)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True, max_steps=40)
    got = chained(m, wl, 2, ipar, rpar)
    assert_same(got, sequential_calls(m, wl, 2, ipar, rpar))
    ierr = got[3].cpu().numpy()
    assert (ierr == -6).any() and (ierr == 1).any()


def test_chain_rejects_bad_arguments():
    from kpp_b200.mechanism import KppError
    m = load("small_strato")
    wl = workloads.for_mechanism(m, "small_strato", 8)
    ipar, rpar = make_controls()
    with pytest.raises(KppError):
        m.rosenbrock_chain(dev(wl.var), dev(wl.fix), dev(wl.temp), dev(wl.tstart), wl.dt, 0,
                           dev(wl.atol), dev(wl.rtol), ipar, rpar)


def test_chain_replays_from_a_cuda_graph():
    """After one call on a stream (which allocates the workspace and queue
    counter), the chained entry captures into a CUDA graph; replays give the
    eager result."""
    m = load("saprc99")
    wl = workloads.for_mechanism(m, "saprc99_classes", 600, seed=8)
    ipar, rpar = make_controls(method="rodas3", scalar_tol=True)
    want = chained(m, wl, 3, ipar, rpar)
    var0 = dev(wl.var)
    var = var0.clone()
    args = (dev(wl.fix), dev(wl.temp), dev(wl.tstart), wl.dt, 3, dev(wl.atol), dev(wl.rtol),
            ipar, rpar)
    kw = dict(cfactor=dev(wl.cfactor), sun=dev(wl.sun))
    s = torch.cuda.Stream()
    box = [None]

    def body():
        var.copy_(var0)
        box[0] = m.rosenbrock_chain(var, *args, **kw, out=box[0])

    with torch.cuda.stream(s):
        body()
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        body()
    for _ in range(2):
        var.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert_same((var, box[0].istatus, box[0].rstatus, box[0].ierr), want)
