"""GPU parity of the Rosenbrock discrete adjoint (kpp_b200_rosenbrock_adj,
int/rosenbrock_adj.c) against the reference's own C RosenbrockADJ.

The device adjoint runs in the library built on KPP's own generator with the
Hessian (libkpp_b200_<mech>_kpproute.so); its host build is bit-identical to
the reference (tests/test_adj_host.py).  On the GPU the arithmetic is the
same operation for operation; the differences are last-ulp ones of the math
library (CUDA's exp/log in the rate constants against glibc's; the
controllers' pow is correctly rounded on the device).  The bar: IERR
identical for every cell, ISTATUS identical for >= 99 % of cells, the final
state within 1e-9 relative above 1e-20 (tests/parity.py's bar without
alternates), and each adjoint vector within ADJ_TOL of its largest entry on
cells that kept the reference's step sequence.  Also: the kppcu library and
the continuous adjoint types refuse the call, and the output arrays keep the
reference's layout.
"""
import ctypes

import numpy as np
import pytest
import torch

from kpp_b200 import KppError, Mechanism, build, workloads

pytestmark = pytest.mark.gpu

ADJ_TOL = 1e-8
BUFSIZE = 800


def dev(a, dtype=torch.float64):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(
        device="cuda", dtype=dtype)


def route(mech):
    path = build.library_path(mech, "kpp")
    if not path.exists():
        pytest.skip(f"{path.name} not built")
    return Mechanism(mech, path=path)


def reference(mech):
    from oracle_lib import REF_DIR
    p = REF_DIR / f"{mech}_adj" / f"libkppadj_{mech}.so"
    if not p.exists():
        pytest.skip("adjoint oracle libraries not present")
    lib = ctypes.CDLL(str(p))
    lib.kppadj_integrate.argtypes = ([ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 9
                                     + [ctypes.c_int] + [ctypes.c_void_p] * 3 + [ctypes.c_int]
                                     + [ctypes.c_void_p] * 3)
    return lib.kppadj_integrate


def controls(method=0, save_lu=False, adjoint=0, autonomous=False):
    ic, rc = [0] * 20, [0.0] * 20
    ic[0] = 1 if autonomous else 0
    ic[1] = 1
    ic[2] = method
    ic[6] = adjoint
    ic[7] = 1 if save_lu else 0
    return ic, rc


def run_both(mech, n, seed, nadj, ic, rc):
    from oracle_lib import OracleLib, quiet_stdout
    m = route(mech)
    ref = reference(mech)
    wl = workloads.for_mechanism(OracleLib(mech), mech, n, seed=seed)
    t0, t1 = wl.step_bounds(0)
    lam0 = np.random.default_rng(seed).standard_normal((nadj * m.nvar, n))
    # the reference, cell by cell on the CPU
    p = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)
    f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
    var_r, lam_r = wl.var.copy(), lam0.copy()
    fix_r = f64(wl.fix) if wl.fix.shape[0] else np.zeros((1, n))
    ist_r, rst_r, ierr_r = np.zeros((8, n), np.int32), np.zeros((3, n)), np.zeros(n, np.int32)
    ic_a, rc_a = np.array(ic, np.int32), np.array(rc, np.float64)
    temp, tt0, tt1 = f64(wl.temp), f64(t0), f64(t1)
    cf, sun, at, rt = f64(wl.cfactor), f64(wl.sun), f64(wl.atol), f64(wl.rtol)
    with quiet_stdout():
        ref(n, n, p(var_r), p(fix_r), p(temp), p(cf), p(sun), p(tt0), p(tt1), p(at), p(rt), nadj,
            p(lam_r), p(ic_a), p(rc_a), BUFSIZE, p(ist_r), p(rst_r), p(ierr_r))
    # the device
    var, lam = dev(wl.var), dev(lam0)
    r = m.rosenbrock_adj(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol),
                         dev(wl.rtol), lam, ic, rc, bufsize=BUFSIZE, cfactor=dev(wl.cfactor),
                         sun=dev(wl.sun))
    torch.cuda.synchronize()
    got = (var.cpu().numpy(), lam.cpu().numpy(), r.istatus.cpu().numpy(),
           r.rstatus.cpu().numpy(), r.ierr.cpu().numpy())
    return got, (var_r, lam_r, ist_r, rst_r, ierr_r), m.nvar


def check(got, ref, nvar, nadj, what):
    var, lam, ist, rst, ierr = got
    var_r, lam_r, ist_r, rst_r, ierr_r = ref
    np.testing.assert_array_equal(ierr, ierr_r, err_msg=what)
    same = np.all(ist == ist_r, axis=0)
    above = np.abs(var_r) > 1e-20
    rel = np.abs(var - var_r)[above] / np.abs(var_r)[above]
    worst_var = float(rel.max()) if rel.size else 0.0
    worst_lam = 0.0
    for m in range(nadj):
        a = lam[m * nvar:(m + 1) * nvar][:, same]
        b = lam_r[m * nvar:(m + 1) * nvar][:, same]
        scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
        if a.size:
            worst_lam = max(worst_lam, float((np.abs(a - b).max(axis=0) / scale).max()))
    print(f"\n[adj bar] {what}: {same.mean():.4f} of {same.size} cells keep the sequence; "
          f"largest relative error of VAR {worst_var:.3g}, of Lambda {worst_lam:.3g}")
    assert same.mean() >= 0.99, what
    assert worst_var <= 1e-9, what
    assert worst_lam <= ADJ_TOL, what
    ok = ierr_r == 1
    np.testing.assert_allclose(rst[0][ok], rst_r[0][ok], rtol=1e-12, err_msg=what)


@pytest.mark.parametrize("mech", ["small_strato", "saprc99"])
@pytest.mark.parametrize("method", [0, 1, 5])
def test_adjoint_matches_reference(mech, method):
    ic, rc = controls(method=method)
    got, ref, nvar = run_both(mech, 256, 71 + method, 2, ic, rc)
    assert (ref[4] == 1).all()
    check(got, ref, nvar, 2, f"{mech} method {method}")


@pytest.mark.parametrize("case", ["save_lu", "autonomous", "forward_only", "rodas3_1"])
def test_adjoint_options_match_reference(case):
    kw = {"save_lu": dict(save_lu=True), "autonomous": dict(autonomous=True),
          "forward_only": dict(adjoint=1), "rodas3_1": dict(method=7)}[case]
    ic, rc = controls(**kw)
    got, ref, nvar = run_both("saprc99", 128, 81, 3, ic, rc)
    check(got, ref, nvar, 3, case)
    if case == "forward_only":
        np.testing.assert_array_equal(got[1], ref[1])  # Lambda untouched


def test_error_returns_and_refusals():
    ic, rc = controls()
    ic[3] = 50  # any ICNTRL[3] != 0: IERR -1 in the reference
    got, ref, nvar = run_both("small_strato", 64, 91, 1, ic, rc)
    assert (got[4] == -1).all() and (ref[4] == -1).all()
    m = route("small_strato")
    wl = workloads.for_mechanism(m, "small_strato", 8, seed=3)
    t0, t1 = wl.step_bounds(0)
    args = (dev(wl.var), dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol),
            dev(wl.rtol), dev(np.zeros((m.nvar, 8))))
    ic, rc = controls(adjoint=3)
    with pytest.raises(KppError):
        m.rosenbrock_adj(*args, ic, rc)
    from kpp_b200 import load
    with pytest.raises(KppError):
        load("small_strato").rosenbrock_adj(*args, *controls())
