"""What the trained scheduler (kpp_b200/schedulers/saprc99_uniform95.npz)
gains over the same integrator without it, on 2^16 fresh saprc99 cells of the
evaluation seed (the training tuples used another seed):
  - fewer internal steps (the proposed Hstart),
  - a predicted cost that ranks the cells' real step counts,
  - a shorter run than the plain launch and than the work queue without the
    network, with the same failure flags."""
from pathlib import Path

import numpy as np
import pytest
import torch

from kpp_b200 import load, workloads
from kpp_b200.scheduler import LearnedScheduler

pytestmark = pytest.mark.gpu

WEIGHTS = Path(__file__).resolve().parents[1] / "kpp_b200" / "schedulers" / "saprc99_uniform95.npz"


def spearman(a, b):
    ra, rb = np.argsort(np.argsort(a)), np.argsort(np.argsort(b))
    return float(np.corrcoef(ra, rb)[0, 1])


def test_trained_scheduler_gains_over_plain():
    assert WEIGHTS.exists(), "trained scheduler weights are part of the package"
    mech = load("saprc99")
    n = 1 << 16
    wl = workloads.for_mechanism(mech, "saprc99_uniform95", n, seed=workloads.SEED_EVAL)
    sch = LearnedScheduler.load(WEIGHTS, mech.nvar)
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    fix, temp, cf, sun = D(wl.fix), D(wl.temp), D(wl.cfactor), D(wl.sun)
    atol, rtol = D(wl.atol), D(wl.rtol)
    t0, t1 = (D(x) for x in wl.step_bounds(0))
    pred = torch.empty(n, 2, dtype=torch.float32, device="cuda")

    def timed(fn, reps=2):
        best, out = None, None
        for _ in range(reps):
            var = D(wl.var)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            out = fn(var)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return best, out

    plain_ms, plain = timed(lambda v: mech.rosenbrock(v, fix, temp, t0, t1, atol, rtol, wl.ipar,
                                                      wl.rpar, cfactor=cf, sun=sun))
    queue_ms, _ = timed(lambda v: mech.rosenbrock_chain(v, fix, temp, t0, wl.dt, 1, atol, rtol,
                                                        wl.ipar, wl.rpar, cfactor=cf, sun=sun))

    def learned_run(v):
        hs, order = sch.plan(v, temp, t0, cfactor=cf, sun=sun, tend=t1, pred=pred)
        return mech.rosenbrock_chain(v, fix, temp, t0, wl.dt, 1, atol, rtol, wl.ipar, wl.rpar,
                                     cfactor=cf, sun=sun, hstart=hs, order=order)

    learned_ms, learned = timed(learned_run)
    nst_plain = plain.istatus[2].cpu().numpy()
    nst_learned = learned.istatus[2].cpu().numpy()
    assert torch.equal(plain.ierr, learned.ierr)
    assert nst_learned.mean() < nst_plain.mean()
    assert spearman(pred[:, 1].cpu().numpy(), np.log(nst_learned)) > 0.8
    assert learned_ms < plain_ms and learned_ms < queue_ms, (learned_ms, plain_ms, queue_ms)
