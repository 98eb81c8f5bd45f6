"""GPU parity: the CUDA path, called through the C ABI, against the reference.

Two references are used: the committed golden fixtures (outputs of the
reference's own KPP-generated C code, tests/golden/make_golden.py) and, where
the prebuilt oracle libraries are present, the reference run live on the
same inputs (oracle/_ref, built by oracle/build_ref.sh).
"""
import numpy as np
import pytest
import torch

from kpp_b200 import make_controls, workloads
from parity import FUNJAC_REL_TOL, REL_TOL, assert_var_parity, max_rel_err, rel_err_funjac

pytestmark = pytest.mark.gpu

MECHS = ["small_strato", "saprc99", "mcm_isoprene"]


def dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def load(mech):
    """The mechanism's library; mechanisms built only on request (see
    kpp_b200.build.ON_REQUEST) are skipped when their library is absent."""
    from kpp_b200 import build, load as _load
    if mech in build.ON_REQUEST and not build.library_path(mech).exists():
        pytest.skip(f"{mech} is built on request: python -m kpp_b200.build {mech}")
    return _load(mech)


def alternates(*a, **k):
    from oracle_lib import alternates as alt
    return alt(*a, **k)


def oracle(mech, opt=""):
    from oracle_lib import OracleLib, lib_path
    if not lib_path(mech, opt).exists():
        pytest.skip("oracle libraries not present")
    return OracleLib(mech, opt)


@pytest.mark.parametrize("mech", MECHS)
def test_fun_jac_rates_match_reference(mech, golden_dir):
    g = np.load(golden_dir / f"funjac_{mech}.npz")
    m = load(mech)
    n = g["var"].shape[1]
    for c in range(n):
        sl = slice(c, c + 1)
        sun = None if g["sun"][c] < 0 else dev(g["sun"][sl])
        rc, vd, jv = m.fun_jac(dev(g["var"][:, sl]), dev(g["fix"][:, sl]), dev(g["temp"][sl]),
                               float(g["time"][c]), cfactor=dev(g["cfactor"][sl]), sun=sun)
        torch.cuda.synchronize()
        # rate constants: every entry on its own (no cancellation inside a rate)
        assert max_rel_err(rc.cpu().numpy()[:, 0], g["rconst"][:, c], floor=1e-300) <= FUNJAC_REL_TOL
        assert rel_err_funjac(vd.cpu().numpy()[:, 0], g["vdot"][:, c]) <= FUNJAC_REL_TOL
        assert rel_err_funjac(jv.cpu().numpy()[:, 0], g["jvs"][:, c]) <= FUNJAC_REL_TOL


def run_chain(m, g, nsteps):
    """Chained chemistry steps with INTEGRATE's warm start (STEPMIN = Hexit)."""
    var = dev(g["var0"])
    n = var.shape[1]
    fix, temp = dev(g["fix"]), dev(g["temp"])
    cf = dev(g["cfactor"]) if g["cfactor"].size else None
    sun = dev(g["sun"]) if g["sun"].size else None
    atol, rtol = dev(g["atol"]), dev(g["rtol"])
    hstart = torch.zeros(n, dtype=torch.float64, device="cuda")
    outs = []
    for k in range(nsteps):
        t0 = dev(g["tstart"] + k * float(g["dt"]))
        t1 = dev(g["tstart"] + (k + 1) * float(g["dt"]))
        r = m.rosenbrock(var, fix, temp, t0, t1, atol, rtol, g["ipar"].tolist(),
                         g["rpar"].tolist(), cfactor=cf, sun=sun, hstart=hstart)
        hstart = r.rstatus[1].clone()
        torch.cuda.synchronize()
        outs.append((var.cpu().numpy().copy(), r.istatus.cpu().numpy(), r.rstatus.cpu().numpy(),
                     r.ierr.cpu().numpy()))
    return outs


@pytest.mark.parametrize("mech", MECHS)
def test_integrate_matches_golden(mech, golden_dir):
    g = np.load(golden_dir / f"integrate_{mech}.npz")
    m = load(mech)
    nsteps = g["var"].shape[0]
    outs = run_chain(m, g, nsteps)
    for k, (var, ist, rst, ierr) in enumerate(outs):
        np.testing.assert_array_equal(ierr, g["ierr"][k])
        assert_var_parity(var, g["var"][k], g["var_alt"][k], f"step {k}")
        same_stats = np.all(ist == g["istatus"][k], axis=0).mean()
        assert same_stats >= 0.95, f"step {k}: ISTATUS equal for {same_stats:.3f} of cells"
        assert max_rel_err(rst[0], g["rstatus"][k][0], floor=0) <= 1e-12


@pytest.mark.parametrize("mech,ncells,nsteps", [("small_strato", 4096, 12), ("saprc99", 512, 1),
                                                ("mcm_isoprene", 64, 1)])
def test_integrate_matches_live_reference(mech, ncells, nsteps):
    o = oracle(mech)
    alt = oracle(mech, "_O3")
    m = load(mech)
    wl = workloads.for_mechanism(m, mech, ncells, seed=7)
    fix_ref = wl.fix if wl.fix.shape[0] else np.zeros((1, ncells))  # the C model pads NFIX
    var_ref = wl.var.copy()
    hs_ref = np.zeros(ncells)
    var = dev(wl.var)
    hstart = torch.zeros(ncells, dtype=torch.float64, device="cuda")
    args = dict(cfactor=None if wl.cfactor is None else dev(wl.cfactor),
                sun=None if wl.sun is None else dev(wl.sun))
    fix, temp, atol, rtol = dev(wl.fix), dev(wl.temp), dev(wl.atol), dev(wl.rtol)
    for k in range(nsteps):
        t0, t1 = wl.step_bounds(k)
        prev = var_ref.copy()
        var_ref, ist, rst, ierr = o.integrate(var_ref, fix_ref, wl.temp, t0, t1, wl.atol, wl.rtol,
                                              wl.ipar, wl.rpar, cfactor=wl.cfactor, sun=wl.sun,
                                              hstart=hs_ref)
        var_alt = alternates(mech, prev, fix_ref, wl.temp, t0, t1, wl.atol, wl.rtol, wl.ipar,
                             wl.rpar, cfactor=wl.cfactor, sun=wl.sun, hstart=hs_ref)
        hs_ref = rst[1].copy()
        r = m.rosenbrock(var, fix, temp, dev(t0), dev(t1), atol, rtol, wl.ipar, wl.rpar,
                         hstart=hstart, **args)
        hstart = r.rstatus[1].clone()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(r.ierr.cpu().numpy(), ierr)
        # saprc99, the benchmark mechanism, needs no rounding envelope at all
        assert_var_parity(var.cpu().numpy(), var_ref, var_alt, f"step {k}",
                          **({"max_env_fraction": 0.0} if mech == "saprc99" else {}))
        assert np.all(r.istatus.cpu().numpy() == ist, axis=0).mean() >= 0.95
        # continue both chains from the reference state so each step is compared
        # from identical inputs
        var.copy_(dev(var_ref))
        hstart.copy_(dev(hs_ref))


@pytest.mark.parametrize("method", ["ros2", "ros3", "ros4", "rodas3", "rodas4"])
def test_every_method_matches_reference(method):
    o = oracle("small_strato")
    m = load("small_strato")
    wl = workloads.for_mechanism(m, "small_strato", 256, seed=11)
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    t0, t1 = wl.step_bounds(0)
    var_ref, ist, rst, ierr = o.integrate(wl.var, wl.fix, wl.temp, t0, t1, wl.atol, wl.rtol, ipar, rpar)
    oracle("small_strato", "_O3")
    var_alt = alternates("small_strato", wl.var, wl.fix, wl.temp, t0, t1, wl.atol, wl.rtol,
                         ipar, rpar)
    var = dev(wl.var)
    r = m.rosenbrock(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol),
                     dev(wl.rtol), ipar, rpar)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r.ierr.cpu().numpy(), ierr)
    assert_var_parity(var.cpu().numpy(), var_ref, var_alt, method)
    assert np.all(r.istatus.cpu().numpy() == ist, axis=0).mean() >= 0.95


def _controls_cases():
    base = dict(method="rodas3", scalar_tol=True)
    return [
        ("bad_method", dict(base, method=0), {}),
        ("bad_method_7", dict(base, method=7), {}),
        ("neg_max_steps", dict(base, max_steps=-1), {}),
        ("neg_hmin", dict(base, hmin=-1.0), {}),
        ("neg_hmax", dict(base, hmax=-1.0), {}),
        ("neg_facmin", dict(base, facmin=-0.5), {}),
        ("neg_facsafe", dict(base, facsafe=-0.5), {}),
        ("tiny_rtol", dict(base), {"rtol": 1e-17}),
        ("zero_atol", dict(base), {"atol": 0.0}),
        ("max_steps_2", dict(base, max_steps=2), {}),
        ("tiny_hmax", dict(base, hmax=1e-300), {}),
        ("vector_tol", dict(method="rodas3", scalar_tol=False), {"vector": True}),
    ]


@pytest.mark.parametrize("name,ctl,tol", _controls_cases(), ids=[c[0] for c in _controls_cases()])
def test_error_codes_and_controls_match_reference(name, ctl, tol):
    o = oracle("small_strato")
    m = load("small_strato")
    wl = workloads.for_mechanism(m, "small_strato", 64, seed=3)
    ipar, rpar = make_controls(**ctl)
    nv = m.nvar
    if tol.get("vector"):
        atol = np.linspace(0.5, 2.0, nv)
        rtol = np.linspace(1e-4, 1e-3, nv)
    else:
        atol = np.array([tol.get("atol", 1.0)])
        rtol = np.array([tol.get("rtol", 1e-3)])
    t0, t1 = wl.step_bounds(0)
    var_ref, ist, rst, ierr = o.integrate(wl.var, wl.fix, wl.temp, t0, t1, atol, rtol, ipar, rpar)
    oracle("small_strato", "_O3")
    var_alt = alternates("small_strato", wl.var, wl.fix, wl.temp, t0, t1, atol, rtol, ipar, rpar)
    var = dev(wl.var)
    r = m.rosenbrock(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(atol), dev(rtol),
                     ipar, rpar)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(r.ierr.cpu().numpy(), ierr)
    assert_var_parity(var.cpu().numpy(), var_ref, var_alt, name)
    assert np.all(r.istatus.cpu().numpy() == ist, axis=0).mean() >= 0.95


def test_empty_and_ragged_batches():
    m = load("small_strato")
    wl = workloads.for_mechanism(m, "small_strato", 37, seed=5)
    # empty batch: a no-op
    z = torch.zeros(m.nvar, 0, dtype=torch.float64, device="cuda")
    e = torch.zeros(0, dtype=torch.float64, device="cuda")
    m.rosenbrock(z, torch.zeros(m.nfix, 0, dtype=torch.float64, device="cuda"), e, e, e,
                 dev(wl.atol), dev(wl.rtol), wl.ipar, wl.rpar, ncells=0)
    # ragged: ncells < ld leaves the padding columns untouched
    ld = 64
    var = torch.full((m.nvar, ld), -7.0, dtype=torch.float64, device="cuda")
    var[:, :37] = dev(wl.var)
    pad = lambda a: np.concatenate([a, np.ones(a.shape[:-1] + (ld - 37,))], axis=-1)
    t0, t1 = wl.step_bounds(0)
    r = m.rosenbrock(var, dev(pad(wl.fix)), dev(pad(wl.temp)), dev(pad(t0)), dev(pad(t1)),
                     dev(wl.atol), dev(wl.rtol), wl.ipar, wl.rpar, ncells=37)
    torch.cuda.synchronize()
    assert torch.all(var[:, 37:] == -7.0)
    assert torch.all(r.ierr[:37] == 1)


def test_singular_pivot_detected():
    """KppDecomp returns k+1 for a zero diagonal on entry to row k."""
    m = load("small_strato")
    irow, icol, crow, diag = m.lu_pattern()
    jvs = torch.zeros(m.lu_nonzero, 4, dtype=torch.float64, device="cuda")
    for d in diag[:-1]:
        jvs[d] = 2.0
    jvs[diag[2], 1] = 0.0
    jvs[diag[0], 3] = 0.0
    ising = m.decomp_solve(jvs)
    torch.cuda.synchronize()
    assert ising.cpu().tolist() == [0, 3, 0, 1]


def test_host_entry_matches_device_entry():
    """kpp_b200_rosenbrock_host (chunked, two streams) gives the device entry's
    results bit for bit, for chunks that do not divide the batch."""
    m = load("saprc99")
    wl = workloads.for_mechanism(m, "saprc99", 1000, seed=21)
    t0, t1 = wl.step_bounds(0)
    var = dev(wl.var)
    r = m.rosenbrock(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol), dev(wl.rtol),
                     wl.ipar, wl.rpar, cfactor=dev(wl.cfactor), sun=dev(wl.sun))
    torch.cuda.synchronize()
    h = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hvar = h(wl.var)
    rh = m.rosenbrock_host(hvar, h(wl.fix), h(wl.temp), h(t0), h(t1), h(wl.atol), h(wl.rtol),
                           wl.ipar, wl.rpar, cfactor=h(wl.cfactor), sun=h(wl.sun), chunk=300)
    np.testing.assert_array_equal(hvar.numpy(), var.cpu().numpy())
    np.testing.assert_array_equal(rh.istatus.numpy(), r.istatus.cpu().numpy())
    np.testing.assert_array_equal(rh.rstatus.numpy(), r.rstatus.cpu().numpy())
    np.testing.assert_array_equal(rh.ierr.numpy(), r.ierr.cpu().numpy())


@pytest.mark.parametrize("method", ["ros2", "ros3", "ros4", "rodas3", "rodas4"])
@pytest.mark.parametrize("sun_mode", ["per_cell", "update_sun"])
def test_warp_kernel_bit_identical_to_thread_kernel(method, sun_mode):
    """The warp-per-cell kernel (work set in shared memory) and the
    thread-per-cell kernel give the same bits: same operations, same order."""
    m = load("saprc99")
    wl = workloads.for_mechanism(m, "saprc99", 300, seed=41)
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    t0, t1 = wl.step_bounds(0)
    sun = dev(wl.sun) if sun_mode == "per_cell" else None
    outs = []
    try:
        for which in ("thread", "warp"):
            m.set_kernel(which)
            assert m.kernel() == which
            var = dev(wl.var)
            r = m.rosenbrock(var, dev(wl.fix), dev(wl.temp), dev(t0), dev(t1), dev(wl.atol),
                             dev(wl.rtol), ipar, rpar, cfactor=dev(wl.cfactor), sun=sun,
                             hstart=dev(np.full(300, 10.0)))
            torch.cuda.synchronize()
            outs.append([var.cpu().numpy(), r.istatus.cpu().numpy(), r.rstatus.cpu().numpy(),
                         r.ierr.cpu().numpy()])
    finally:
        m.set_kernel("auto")
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("mech", MECHS)
def test_shuffle_entries_follow_the_species_map(mech):
    m = load(mech)
    idx = m.user_species()
    n, nuser = 300, len(idx)
    vu = torch.rand(nuser, n, dtype=torch.float64, device="cuda")
    var = torch.full((m.nvar, n), -1.0, dtype=torch.float64, device="cuda")
    m.shuffle_user2kpp(vu, var)
    back = torch.full((nuser, n), -7.0, dtype=torch.float64, device="cuda")
    m.shuffle_kpp2user(var, back)
    torch.cuda.synchronize()
    want = np.full((m.nvar, n), -1.0)
    wback = np.full((nuser, n), -7.0)
    vu_h = vu.cpu().numpy()
    for k, f in enumerate(idx):
        if f >= 0:
            want[f] = vu_h[k]
            wback[k] = vu_h[k]
    np.testing.assert_array_equal(var.cpu().numpy(), want)
    np.testing.assert_array_equal(back.cpu().numpy(), wback)
