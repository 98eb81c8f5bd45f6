"""The three integrators at the benchmark's full size: 2^20 saprc99 cells of
the benchmark workload (uniform solar zenith angles, one 600 s chemistry
step), through properties that do not depend on the batch size:

  * every cell succeeds (IERR = 1);
  * 256 cells spread over the batch give, bit for bit, what the same cells
    give integrated alone (nothing in a cell's result depends on the other
    2^20 - 1 cells, on its position or on the work arrays' reuse);
  * those cells meet the parity bar against the reference's own C
    integrator, live, with its rounding alternates.
"""
import numpy as np
import pytest
import torch

from kpp_b200 import workloads

pytestmark = pytest.mark.gpu

N = 1 << 20
SAMPLE = np.linspace(0, N - 1, 256).astype(np.int64)


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def _run(m, integ, wl, idx, ic, rc):
    """The integrator on the cells `idx` of the workload (None: all)."""
    sel = (lambda a: a) if idx is None else (lambda a: a[..., idx])
    var = dev(sel(wl.var))
    t0, t1 = wl.step_bounds(0)
    args = (var, dev(sel(wl.fix)), dev(sel(wl.temp)), dev(sel(t0)), dev(sel(t1)),
            dev(wl.atol), dev(wl.rtol), ic, rc)
    kw = dict(cfactor=dev(sel(wl.cfactor)), sun=dev(sel(wl.sun)))
    if integ == "rosenbrock":
        r = m.rosenbrock(*args, **kw)
    elif integ == "sdirk":
        r = m.sdirk(*args, **kw)
    else:
        r = m.runge_kutta(*args, **kw)
    torch.cuda.synchronize()
    out = [x.cpu().numpy() for x in (var, r.istatus, r.rstatus, r.ierr)]
    del var, r
    torch.cuda.empty_cache()
    return out


@pytest.mark.parametrize("integ", ["rosenbrock", "sdirk", "rk"])
def test_full_size_batch_properties(integ):
    from kpp_b200 import load
    m = load("saprc99")
    wl = workloads.for_mechanism(m, "saprc99_uniform95", N)
    if integ == "rosenbrock":
        ic, rc = wl.ipar, wl.rpar  # Rodas3, the benchmark's controls
    elif integ == "sdirk":
        from test_gpu_sdirk import controls
        ic, rc = controls(method=5)
    else:
        from test_rk_host import rk_controls
        ic, rc = rk_controls(method=0)

    full = _run(m, integ, wl, None, ic, rc)
    assert (full[3] == 1).all(), f"{integ}: {(full[3] != 1).sum()} cells failed"
    alone = _run(m, integ, wl, SAMPLE, ic, rc)
    for a, b in zip(full, alone):
        np.testing.assert_array_equal(a[..., SAMPLE], b)

    # the sample against the reference, live
    t0, t1 = wl.step_bounds(0)
    s = lambda a: np.ascontiguousarray(a[..., SAMPLE])
    cells = (s(wl.var), s(wl.fix), s(wl.temp), s(t0), s(t1), wl.atol, wl.rtol, ic, rc)
    kw = dict(cfactor=s(wl.cfactor), sun=s(wl.sun))
    if integ == "rosenbrock":
        from oracle_lib import OracleLib, alternates, lib_path
        from parity import assert_var_parity
        if not lib_path("saprc99", "_O3").exists():
            pytest.skip("oracle libraries not present")
        ref = OracleLib("saprc99").integrate(*cells, **kw)
        alt = alternates("saprc99", *cells, **kw)
        np.testing.assert_array_equal(alone[3], ref[3])
        assert_var_parity(alone[0], ref[0], alt, "rosenbrock 2^20")
        assert np.all(alone[1] == ref[1], axis=0).mean() >= 0.95
    elif integ == "sdirk":
        from oracle_lib import SdirkOracle, sdirk_alternates, sdirk_lib_path
        from test_gpu_sdirk import check
        if not sdirk_lib_path("saprc99", "_pw").exists():
            pytest.skip("SDIRK oracle libraries not present")
        ref = SdirkOracle("saprc99").integrate(*cells, **kw)
        check(alone, ref, sdirk_alternates("saprc99", *cells, **kw), "sdirk 2^20")
    else:
        from oracle_lib import RkOracle, rk_alternates, rk_lib_path
        from test_gpu_rk import check
        if not rk_lib_path("saprc99", "_pw").exists():
            pytest.skip("Runge-Kutta oracle libraries not present")
        ref = RkOracle("saprc99").integrate(*cells, **kw)
        check(alone, ref, rk_alternates("saprc99", *cells, **kw), "rk 2^20", wl.atol, wl.rtol)
