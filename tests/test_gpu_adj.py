"""GPU parity of the Rosenbrock discrete adjoint (kpp_b200_rosenbrock_adj,
int/rosenbrock_adj.c) against the reference's own C RosenbrockADJ.

The device adjoint runs in the library built on KPP's own generator with the
Hessian (libkpp_b200_<mech>_kpproute.so); its host build is bit-identical to
the reference (tests/test_adj_host.py).  On the GPU the arithmetic is the
same operation for operation; the differences are last-ulp ones of the math
library (CUDA's exp/log in the rate constants against glibc's; the
controllers' pow is correctly rounded on the device).  The adjoint amplifies
such perturbations: each backward step solves with (I/(h gamma) - J)^T, whose
condition number on saprc99 reaches ~1e11, so the reference itself, compiled
with FMA contraction (libkppadj_<mech>_O3.so: another valid rounding of the
same code), moves Lambda by up to ~5e-5 of its largest entry while VAR moves
by ~1e-11.  The bar: IERR identical for every cell, ISTATUS identical for
>= 99 % of cells, the final state within tests/parity.py's bar (1e-9
relative above 1e-20, or ILL_FACTOR times the FMA build's distance from the
reference), and, on cells that kept the reference's step sequence, each
cell's adjoint vectors within max(ADJ_TOL, ILL_FACTOR x the FMA build's
distance) of the reference, relative to the cell's largest entry, taken
over the cells: for the largest and for the median per-cell distance (the
perturbation a cell receives differs between the two roundings, so the bar
compares the distributions, not cell by cell).  Also: the
kppcu library and the continuous adjoint types refuse the call, and the
output arrays keep the reference's layout.
"""
import ctypes

import numpy as np
import pytest
import torch

from kpp_b200 import KppError, Mechanism, build, workloads
from parity import ILL_FACTOR, var_parity

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


def reference(mech, suffix=""):
    from oracle_lib import REF_DIR
    p = REF_DIR / f"{mech}_adj" / f"libkppadj_{mech}{suffix}.so"
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
    wl = workloads.for_mechanism(OracleLib(mech), mech, n, seed=seed)
    t0, t1 = wl.step_bounds(0)
    lam0 = np.random.default_rng(seed).standard_normal((nadj * m.nvar, n))
    # the reference, cell by cell on the CPU: its -O build, and its FMA build
    # (the reference's own rounding spread)
    p = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)
    f64 = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
    fix_r = f64(wl.fix) if wl.fix.shape[0] else np.zeros((1, n))
    ic_a, rc_a = np.array(ic, np.int32), np.array(rc, np.float64)
    temp, tt0, tt1 = f64(wl.temp), f64(t0), f64(t1)
    cf, sun, at, rt = f64(wl.cfactor), f64(wl.sun), f64(wl.atol), f64(wl.rtol)
    runs = []
    for suffix in ("", "_O3"):
        ref = reference(mech, suffix)
        var_r, lam_r = wl.var.copy(), lam0.copy()
        ist_r, rst_r, ierr_r = np.zeros((8, n), np.int32), np.zeros((3, n)), np.zeros(n, np.int32)
        with quiet_stdout():
            ref(n, n, p(var_r), p(fix_r), p(temp), p(cf), p(sun), p(tt0), p(tt1), p(at), p(rt),
                nadj, p(lam_r), p(ic_a), p(rc_a), BUFSIZE, p(ist_r), p(rst_r), p(ierr_r))
        runs.append((var_r, lam_r, ist_r, rst_r, ierr_r))
    # the device
    var, lam = dev(wl.var), dev(lam0)
    r = m.rosenbrock_adj(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol),
                         dev(wl.rtol), lam, ic, rc, bufsize=BUFSIZE, cfactor=dev(wl.cfactor),
                         sun=dev(wl.sun))
    torch.cuda.synchronize()
    got = (var.cpu().numpy(), lam.cpu().numpy(), r.istatus.cpu().numpy(),
           r.rstatus.cpu().numpy(), r.ierr.cpu().numpy())
    return got, runs[0], m.nvar, runs[1]


def check(got, ref, nvar, nadj, what, alt):
    var, lam, ist, rst, ierr = got
    var_r, lam_r, ist_r, rst_r, ierr_r = ref
    np.testing.assert_array_equal(ierr, ierr_r, err_msg=what)
    same = np.all(ist == ist_r, axis=0) & np.all(alt[2] == ist_r, axis=0)
    pv = var_parity(var, var_r, alt[0])
    # per cell: distance of each adjoint vector from the reference's,
    # relative to the vector's largest entry, for the device and for the
    # reference's FMA build
    errs, spreads = [], []
    for m in range(nadj):
        a = lam[m * nvar:(m + 1) * nvar][:, same]
        b = lam_r[m * nvar:(m + 1) * nvar][:, same]
        c = alt[1][m * nvar:(m + 1) * nvar][:, same]
        if not a.size:
            continue
        scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
        errs.append(np.abs(a - b).max(axis=0) / scale)
        spreads.append(np.abs(c - b).max(axis=0) / scale)
    err = np.concatenate(errs) if errs else np.zeros(1)
    spread = np.concatenate(spreads) if spreads else np.zeros(1)
    ratio_max = float(err.max() / max(ADJ_TOL, ILL_FACTOR * float(spread.max())))
    ratio_med = float(np.median(err) / max(ADJ_TOL, ILL_FACTOR * float(np.median(spread))))
    print(f"\n[adj bar] {what}: {same.mean():.4f} of {same.size} cells keep the sequence; "
          f"VAR: largest relative error {pv['well']:.3g} (FMA-build envelope ratio "
          f"{pv['ratio']:.3g}, {pv['n_env']} entries beyond 1e-9); Lambda per cell, of its "
          f"largest entry: device largest {err.max():.3g} median {np.median(err):.3g}, the "
          f"reference's FMA build largest {spread.max():.3g} median {np.median(spread):.3g}; "
          f"ratios to the bar {ratio_max:.3g} / {ratio_med:.3g}")
    assert same.mean() >= 0.99, what
    assert pv["ratio"] <= 1.0, what
    assert ratio_max <= 1.0 and ratio_med <= 1.0, what
    ok = ierr_r == 1
    np.testing.assert_allclose(rst[0][ok], rst_r[0][ok], rtol=1e-12, err_msg=what)


@pytest.mark.parametrize("mech", ["small_strato", "saprc99"])
@pytest.mark.parametrize("method", [0, 1, 5])
def test_adjoint_matches_reference(mech, method):
    ic, rc = controls(method=method)
    got, ref, nvar, alt = run_both(mech, 256, 71 + method, 2, ic, rc)
    assert (ref[4] == 1).all()
    check(got, ref, nvar, 2, f"{mech} method {method}", alt)


@pytest.mark.parametrize("case", ["save_lu", "autonomous", "forward_only", "rodas3_1"])
def test_adjoint_options_match_reference(case):
    kw = {"save_lu": dict(save_lu=True), "autonomous": dict(autonomous=True),
          "forward_only": dict(adjoint=1), "rodas3_1": dict(method=7)}[case]
    ic, rc = controls(**kw)
    got, ref, nvar, alt = run_both("saprc99", 128, 81, 3, ic, rc)
    check(got, ref, nvar, 3, case, alt)
    if case == "forward_only":
        np.testing.assert_array_equal(got[1], ref[1])  # Lambda untouched


def test_error_returns_and_refusals():
    ic, rc = controls()
    ic[3] = 50  # any ICNTRL[3] != 0: IERR -1 in the reference
    got, ref, nvar, _ = run_both("small_strato", 64, 91, 1, ic, rc)
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
