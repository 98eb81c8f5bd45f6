"""GPU parity of the SDIRK integrator (int/sdirk.c of the reference) against
the reference's own C SDIRK on the same generated model.

The reference is the mechanism generated with `#INTEGRATOR sdirk` and driven
cell by cell (oracle/refkpp/batch_driver_sdirk.c).  The bar is the one of the
Rosenbrock path: identical return value per cell, concentrations within
1e-9 relative (or within the reference's own spread under valid last-ulp
roundings: FMA contraction, SUN one ulp up / down, the integrator's pow()
one ulp up / down), and the same integrator
statistics ISTATUS[1..8] for almost every cell.
"""
import numpy as np
import pytest
import torch

from kpp_b200 import workloads
from parity import assert_var_parity, max_rel_err

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def oracle(mech):
    from oracle_lib import SdirkOracle, sdirk_lib_path
    for opt in ("", "_O3", "_pw"):
        if not sdirk_lib_path(mech, opt).exists():
            pytest.skip("SDIRK oracle libraries not present")
    return SdirkOracle(mech)


def controls(method=0, scalar_tol=True, **kw):
    """ICNTRL / RCNTRL in the C layout of int/sdirk.c (ICNTRL[1] = ITOL
    switch, [2] method, [3] max steps, [4] Newton iterations, [5] Newton start
    guess; RCNTRL[0..10] Hmin, Hmax, Hstart, FacMin, FacMax, FacRej, FacSafe,
    ThetaMin, NewtonTol, Qmin, Qmax)."""
    ic = [0] * 20
    rc = [0.0] * 20
    ic[1] = 1 if scalar_tol else 0
    ic[2] = method
    for k, v in kw.items():
        slot = {"max_steps": (ic, 3), "newton_maxit": (ic, 4), "start_newton": (ic, 5),
                "hmin": (rc, 0), "hmax": (rc, 1), "hstart": (rc, 2), "facmin": (rc, 3),
                "facmax": (rc, 4), "facrej": (rc, 5), "facsafe": (rc, 6), "theta_min": (rc, 7),
                "newton_tol": (rc, 8), "qmin": (rc, 9), "qmax": (rc, 10)}[k]
        slot[0][slot[1]] = v
    return ic, rc


def run_both(mech, ncells, seed, ic, rc, atol=None, rtol=None, step=0, var0=None):
    from kpp_b200 import load
    from oracle_lib import sdirk_alternates
    o = oracle(mech)
    m = load(mech)
    wl = workloads.for_mechanism(m, mech, ncells, seed=seed)
    atol = wl.atol if atol is None else atol
    rtol = wl.rtol if rtol is None else rtol
    var0 = wl.var if var0 is None else var0
    fix_ref = wl.fix if wl.fix.shape[0] else np.zeros((1, ncells))  # the C model pads NFIX
    t0, t1 = wl.step_bounds(step)
    ref = o.integrate(var0, fix_ref, wl.temp, t0, t1, atol, rtol, ic, rc, cfactor=wl.cfactor,
                      sun=wl.sun)
    alt = sdirk_alternates(mech, var0, fix_ref, wl.temp, t0, t1, atol, rtol, ic, rc,
                           cfactor=wl.cfactor, sun=wl.sun)
    var = dev(var0)
    r = m.sdirk(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(atol), dev(rtol), ic, rc,
                cfactor=None if wl.cfactor is None else dev(wl.cfactor),
                sun=None if wl.sun is None else dev(wl.sun))
    torch.cuda.synchronize()
    got = (var.cpu().numpy(), r.istatus.cpu().numpy(), r.rstatus.cpu().numpy(),
           r.ierr.cpu().numpy())
    return got, ref, alt


def check(got, ref, alt, what, stats_frac=0.99):
    var, ist, rst, ierr = got
    var_ref, ist_ref, rst_ref, ierr_ref = ref
    np.testing.assert_array_equal(ierr, ierr_ref, err_msg=what)
    assert_var_parity(var, var_ref, alt, what)
    same = np.all(ist == ist_ref, axis=0).mean()
    print(f"\n[sdirk bar] {what}: {same:.4f} of {ist.shape[1]} cells with the reference's "
          f"statistics")
    assert same >= stats_frac, what
    ok = ierr_ref == 1
    # Texit: the final time of every successful cell
    assert max_rel_err(rst[0][ok], rst_ref[0][ok], floor=0) <= 1e-12, what


@pytest.mark.parametrize("method", [0, 1, 2, 3, 4, 5, 7])
def test_every_sdirk_method_matches_reference(method):
    ic, rc = controls(method=method)
    got, ref, alt = run_both("small_strato", 512, 11, ic, rc)
    assert (ref[3] == 1).all()
    check(got, ref, alt, f"method {method}")


@pytest.mark.parametrize("step", [0, 3, 6])
def test_sdirk_diurnal_steps_match_reference(step):
    ic, rc = controls(method=3)
    got, ref, alt = run_both("small_strato", 2048, 5, ic, rc, step=step)
    check(got, ref, alt, f"step {step}")


@pytest.mark.parametrize("method", [1, 3, 5])
def test_sdirk_saprc99_matches_reference(method):
    ic, rc = controls(method=method)
    got, ref, alt = run_both("saprc99", 256, 7, ic, rc)
    check(got, ref, alt, f"saprc99 method {method}")


@pytest.mark.parametrize("method", [1, 5])
def test_sdirk_mcm_matches_reference(method):
    from kpp_b200 import build
    if not build.library_path("mcm_isoprene").exists():
        pytest.skip("mcm_isoprene is built on request: python -m kpp_b200.build mcm_isoprene")
    ic, rc = controls(method=method)
    got, ref, alt = run_both("mcm_isoprene", 64, 7, ic, rc)
    check(got, ref, alt, f"mcm method {method}")


def _controls_cases():
    return [
        ("max_steps_3", dict(max_steps=3), {}),
        ("neg_max_steps", dict(max_steps=-1), {}),
        ("newton_maxit_1", dict(newton_maxit=1), {}),
        ("newton_start_zero", dict(start_newton=1), {}),
        ("neg_hmin", dict(hmin=-1.0), {}),
        ("neg_hmax", dict(hmax=-1.0), {}),
        ("hstart", dict(hstart=10.0), {}),
        ("neg_facmin", dict(facmin=-0.5), {}),
        ("facmax_2", dict(facmax=2.0), {}),
        ("theta_min_neg", dict(theta_min=-1.0), {}),
        ("theta_min_2", dict(theta_min=2.0), {}),
        ("newton_tol_big", dict(newton_tol=2.0), {}),
        ("qmin_qmax", dict(qmin=0.5, qmax=2.0), {}),
        ("tiny_rtol", dict(), {"rtol": 1e-17}),
        ("zero_atol", dict(), {"atol": 0.0}),
        ("tiny_hmax", dict(hmax=1e-300), {}),
        ("vector_tol", dict(scalar_tol=False), {"vector": True}),
    ]


@pytest.mark.parametrize("name,ctl,tol", _controls_cases(), ids=[c[0] for c in _controls_cases()])
def test_sdirk_error_codes_and_controls_match_reference(name, ctl, tol):
    from kpp_b200 import load
    nv = load("small_strato").nvar
    ic, rc = controls(method=ctl.pop("method", 3), **ctl)
    if tol.get("vector"):
        atol = np.linspace(0.5, 2.0, nv)
        rtol = np.linspace(1e-4, 1e-3, nv)
    else:
        atol = np.array([tol.get("atol", 1.0)])
        rtol = np.array([tol.get("rtol", 1e-3)])
    got, ref, alt = run_both("small_strato", 64, 3, ic, rc, atol=atol, rtol=rtol)
    check(got, ref, alt, name)


def test_sdirk_empty_and_ragged_batches():
    from kpp_b200 import load
    m = load("small_strato")
    ic, rc = controls(method=3)
    z = torch.zeros(0, dtype=torch.float64, device="cuda")
    r = m.sdirk(torch.zeros(m.nvar, 0, dtype=torch.float64, device="cuda"),
                torch.zeros(m.nfix, 0, dtype=torch.float64, device="cuda"), z, z, z,
                dev(np.array([1.0])), dev(np.array([1e-3])), ic, rc)
    assert r.ierr.numel() == 0
    # a batch that is not a multiple of the warp or block size
    got, ref, alt = run_both("small_strato", 37, 13, ic, rc)
    check(got, ref, alt, "ragged 37")
    # ncells < ld leaves the padding columns untouched
    wl = workloads.for_mechanism(m, "small_strato", 37, seed=13)
    ld = 64
    var = torch.full((m.nvar, ld), -7.0, dtype=torch.float64, device="cuda")
    var[:, :37] = dev(wl.var)
    pad = lambda a: np.concatenate([a, np.ones(a.shape[:-1] + (ld - 37,))], axis=-1)
    t0, t1 = wl.step_bounds(0)
    r = m.sdirk(var, dev(pad(wl.fix)), dev(pad(wl.temp)), dev(pad(t0)), dev(pad(t1)),
                dev(wl.atol), dev(wl.rtol), ic, rc, ncells=37)
    torch.cuda.synchronize()
    assert torch.all(var[:, 37:] == -7.0)
    np.testing.assert_array_equal(var[:, :37].cpu().numpy(), got[0])
    assert torch.all(r.ierr[:37] == 1)


@pytest.mark.parametrize("newton_maxit", [1, 2])
@pytest.mark.parametrize("mech,ncells", [("small_strato", 8192), ("saprc99", 2048)])
def test_sdirk_cell_results_independent_of_batch(mech, ncells, newton_maxit):
    """A cell's result depends on nothing but its own inputs: not on the other
    cells of the batch, their order, or what an earlier launch left in the
    work arrays.  Exercised on the Newton-failure path (one or two Newton
    iterations allowed: most cells fail, or all succeed after rejected
    steps), whose error estimate reads stage vectors of earlier steps."""
    from kpp_b200 import load
    m = load(mech)
    wl = workloads.for_mechanism(m, mech, ncells, seed=21)
    ic, rc = controls(method=4, newton_maxit=newton_maxit)
    t0, t1 = wl.step_bounds(0)
    cf = None if wl.cfactor is None else dev(wl.cfactor)
    sun = None if wl.sun is None else dev(wl.sun)

    def run(idx):
        sel = lambda a: None if a is None else a[..., idx]
        var = dev(wl.var[:, idx])
        r = m.sdirk(var, dev(wl.fix[:, idx]), dev(wl.temp[idx]), dev(t0[idx]), dev(t1[idx]),
                    dev(wl.atol), dev(wl.rtol), ic, rc, cfactor=sel(cf), sun=sel(sun))
        torch.cuda.synchronize()
        return [x.cpu().numpy() for x in (var, r.istatus, r.rstatus, r.ierr)]

    full = run(np.arange(ncells))
    again = run(np.arange(ncells))
    rng = np.random.default_rng(5)
    sub = rng.permutation(ncells)[: ncells // 3]
    part = run(sub)
    for a, b, c in zip(full, again, part):
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(a[..., sub], c)
    assert full[1][4].sum() > 0  # rejected steps: the path was taken


@pytest.mark.parametrize("mech,ncells", [("small_strato", 1000), ("saprc99", 600)])
def test_sdirk_host_entry_matches_device_entry(mech, ncells):
    """kpp_b200_sdirk_host (host arrays, chunks of 256 cells: several chunks
    and a ragged last one; ld > ncells) gives the device entry's results bit
    for bit."""
    from kpp_b200 import load
    m = load(mech)
    wl = workloads.for_mechanism(m, mech, ncells, seed=4)
    ic, rc = controls(method=3)
    t0, t1 = wl.step_bounds(0)
    var = dev(wl.var)
    cf = None if wl.cfactor is None else dev(wl.cfactor)
    sun = None if wl.sun is None else dev(wl.sun)
    r = m.sdirk(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol), dev(wl.rtol), ic,
                rc, cfactor=cf, sun=sun)
    torch.cuda.synchronize()
    ld = ncells + 24
    pad = lambda a: torch.from_numpy(np.ascontiguousarray(np.concatenate(
        [a, np.ones(a.shape[:-1] + (ld - ncells,))], axis=-1))).pin_memory()
    hvar = pad(wl.var)
    hr = m.sdirk_host(hvar, pad(wl.fix), pad(wl.temp), pad(t0), pad(t1),
                      torch.from_numpy(wl.atol), torch.from_numpy(wl.rtol), ic, rc,
                      cfactor=None if wl.cfactor is None else pad(wl.cfactor),
                      sun=None if wl.sun is None else pad(wl.sun), ncells=ncells, chunk=256)
    np.testing.assert_array_equal(hvar[:, :ncells].numpy(), var.cpu().numpy())
    np.testing.assert_array_equal(hr.istatus[:, :ncells].numpy(), r.istatus.cpu().numpy())
    np.testing.assert_array_equal(hr.rstatus[:, :ncells].numpy(), r.rstatus.cpu().numpy())
    np.testing.assert_array_equal(hr.ierr[:ncells].numpy(), r.ierr.cpu().numpy())
    assert torch.all(hvar[:, ncells:] == 1.0)
