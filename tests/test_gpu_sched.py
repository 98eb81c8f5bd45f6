"""The learned scheduler's kernels (libkpp_b200_sched.so) against the CPU
oracle oracle/mlp_oracle.py, and the scheduling pass's contract."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from kpp_b200 import load, workloads
from kpp_b200 import scheduler as S

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu

# FP32 accumulation on the device against float64 in the oracle; the BF16
# rounding points are the same, so only rare rounding flips of a stored BF16
# value separate them.
GRAD_REL_TOL = 2e-3
OUT_REL_TOL = 2e-3


def small_net(nin=20, width=64, nhidden=3, seed=11, batch=300):
    m = S.Mlp(nin, width=width, nhidden=nhidden, nout=2, max_batch=1024)
    m.set_params(S.init_params(nin, width, nhidden, 2, seed))
    rng = np.random.default_rng(seed)
    x = mo.bf16(rng.normal(size=(batch, nin)))
    y = rng.normal(size=(batch, 2)).astype(np.float32)
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to(torch.bfloat16).cuda()
    return m, x, y, xd


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_oracle():
    m, x, _, xd = small_net()
    out = m.forward(xd).cpu().numpy()
    want, _ = mo.forward(m.params_bf16(), m.shapes(), x)
    assert rel(out, want) <= OUT_REL_TOL


@pytest.mark.parametrize("width,batch", [(64, 300), (256, 1024)])
def test_gradients_match_oracle(width, batch):
    m, x, y, xd = small_net(nin=78, width=width, batch=batch)
    loss = float(m.loss_grad(xd, torch.from_numpy(y).cuda()).item())
    g = m.grads()
    want_loss, want_g = mo.loss_grad(m.params_bf16(), m.shapes(), x, y)
    assert abs(loss - want_loss) <= 1e-4 * want_loss
    off = 0
    for fo, fi in m.shapes():
        for k, nm in ((fo * fi, "W"), (fo, "b")):
            assert rel(g[off:off + k], want_g[off:off + k]) <= GRAD_REL_TOL, (nm, fo, fi)
            off += k


def test_adam_step_matches_oracle():
    m, x, y, xd = small_net()
    w0 = m.params().astype(np.float64)
    m.loss_grad(xd, torch.from_numpy(y).cuda())
    g = m.grads().astype(np.float64)
    m.adam(1e-3)
    torch.cuda.synchronize()
    want, _, _ = mo.adam(w0, g, np.zeros_like(w0), np.zeros_like(w0), 1, 1e-3)
    np.testing.assert_allclose(m.params(), want, rtol=2e-6, atol=1e-7)


def test_training_fits_a_smooth_function():
    nin = 8
    m = S.Mlp(nin, width=64, nhidden=3, nout=2, max_batch=512)
    m.set_params(S.init_params(nin, 64, 3, 2, seed=2))
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, size=(4096, nin))
    y = np.stack([np.sin(2 * x[:, 0]) + x[:, 1] * x[:, 2], np.cos(x[:, 3] + x[:, 4])], 1)
    y = ((y - y.mean(0)) / y.std(0)).astype(np.float32)
    X = torch.from_numpy(np.ascontiguousarray(x.T)).to(torch.bfloat16).cuda()
    Y = torch.from_numpy(y).cuda()
    Xb = torch.empty(nin, 512, dtype=torch.bfloat16, device="cuda")
    losses = []
    for step in range(600):
        idx = torch.randint(0, 4096, (512,), device="cuda", dtype=torch.int32)
        S.gather_columns(X, idx, Xb)
        losses.append(float(m.loss_grad(Xb, Y.index_select(0, idx)).item()))
        m.adam(3e-3)
    assert np.mean(losses[-50:]) < 0.1 * np.mean(losses[:10])


def test_features_match_host_definition():
    mech = load("saprc99")
    wl = workloads.for_mechanism(mech, "saprc99_uniform95", 500, seed=9)
    nin = mech.nvar + 4
    f = S.host_features(wl.var, wl.temp, wl.cfactor, wl.sun, wl.dt)
    mu, sd = f.mean(1), f.std(1) + 1e-3
    m = S.Mlp(nin, width=32, nhidden=1)
    m.set_scaling(mu, sd, [0.0, 0.0], [1.0, 1.0])
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    x = m.features(mech.nvar, D(wl.var), D(wl.temp), D(wl.cfactor), D(wl.sun), D(wl.tstart),
                   dt=wl.dt)
    want = mo.bf16((f - mu[:, None]) / sd[:, None])
    got = x.to(torch.float64).cpu().numpy()
    assert np.abs(got - want).max() <= 1e-2 * max(1.0, np.abs(want).max())


def random_scheduler(nvar, seed=4):
    """A scheduler with random weights: its predictions are arbitrary, which
    is all the contract tests need."""
    nin = nvar + 4
    m = S.Mlp(nin)
    m.set_params(S.init_params(nin, S.WIDTH, S.NHIDDEN, S.NOUT, seed))
    mu, sd = np.zeros(nin), np.full(nin, 10.0)
    m.set_scaling(mu, sd, [-4.0, 3.8], [1.0, 0.3])
    return S.LearnedScheduler(m, nvar, mu, sd, np.array([-4.0, 3.8]), np.array([1.0, 0.3]),
                              hmin=1e-6, hmax=1e-2, nbins=256, lnn_lo=2.0, lnn_hi=5.5)


def test_plan_gives_a_cost_sorted_permutation():
    mech = load("saprc99")
    n = 3000
    wl = workloads.for_mechanism(mech, "saprc99_uniform95", n, seed=10)
    sch = random_scheduler(mech.nvar)
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pred = torch.empty(n, 2, dtype=torch.float32, device="cuda")
    hs, order = sch.plan(D(wl.var), D(wl.temp), D(wl.tstart), cfactor=D(wl.cfactor),
                         sun=D(wl.sun), dt=wl.dt, pred=pred)
    torch.cuda.synchronize()
    o = order.cpu().numpy()
    assert np.array_equal(np.sort(o), np.arange(n))
    p = pred.cpu().numpy().astype(np.float64)
    np.testing.assert_allclose(hs.cpu().numpy(), np.clip(10.0 ** p[:, 0], 1e-6, 1e-2), rtol=1e-6)
    b = np.clip(np.floor((5.5 - p[:, 1]) / 3.5 * 256), 0, 255)
    # most expensive bins first (a value on a bin edge may land on either side)
    assert np.all(np.diff(b[o]) >= -1) and np.mean(np.diff(b[o]) >= 0) > 0.99


@pytest.mark.parametrize("mech_name,wname", [("saprc99", "saprc99_uniform95"),
                                             ("small_strato", "small_strato")])
def test_scheduled_run_equals_plain_call_with_the_same_hstart(mech_name, wname):
    """Scheduling changes the order of work and the starting step only: each
    cell's result is the plain entry's for the Hstart the plan chose, and the
    failure flags of the default run are unchanged."""
    mech = load(mech_name)
    n = 2000
    wl = workloads.for_mechanism(mech, wname, n, seed=12)
    sch = random_scheduler(mech.nvar)
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    cf = D(wl.cfactor) if wl.cfactor is not None else None
    sun = D(wl.sun) if wl.sun is not None else None
    t0, t1 = (D(x) for x in wl.step_bounds(0))
    hs, order = sch.plan(D(wl.var), D(wl.temp), t0, cfactor=cf, sun=sun, tend=t1)
    va, vb, vc = D(wl.var), D(wl.var), D(wl.var)
    ipar, rpar = wl.ipar, wl.rpar
    ra = mech.rosenbrock_chain(va, D(wl.fix), D(wl.temp), t0, wl.dt, 1, D(wl.atol), D(wl.rtol),
                               ipar, rpar, cfactor=cf, sun=sun, hstart=hs, order=order)
    rb = mech.rosenbrock(vb, D(wl.fix), D(wl.temp), t0, t1, D(wl.atol), D(wl.rtol), ipar, rpar,
                         cfactor=cf, sun=sun, hstart=hs)
    rc = mech.rosenbrock(vc, D(wl.fix), D(wl.temp), t0, t1, D(wl.atol), D(wl.rtol), ipar, rpar,
                         cfactor=cf, sun=sun)
    torch.cuda.synchronize()
    assert torch.equal(va, vb) and torch.equal(ra.istatus, rb.istatus)
    assert torch.equal(ra.rstatus, rb.rstatus) and torch.equal(ra.ierr, rb.ierr)
    assert torch.equal(ra.ierr, rc.ierr)
