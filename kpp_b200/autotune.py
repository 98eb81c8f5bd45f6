"""Launch-shape autotuner for the batched Rosenbrock kernels.

  python -m kpp_b200.autotune --mech saprc99 --workload saprc99_uniform95

Measures, on a sample of the workload on the current GPU, every candidate
launch shape of the integration: the kernel (one thread per cell, or one
warp per cell where the mechanism has the shared-memory form) and, for the
thread kernel, the number of 128-thread blocks kept resident per SM and, on
the work-queue path, the queue's granularity (32 cells per warp, or one cell
per lane with the lanes' cells advancing step by step together).  Each
candidate runs the same cells the way the benchmark does (the learned
scheduler's plan and the work-queue launch when trained weights exist, the
plain launch otherwise); all candidates must give bit-identical results.
The fastest shape is written to kpp_b200/tuning/<gpu>_<mech>_<workload>.json
with the whole table; `apply()` reads it back.  Results never depend on the
shape, only the time does.
"""
from __future__ import annotations

import argparse
import json
import re
from pathlib import Path
from typing import Optional

import numpy as np
import torch

from . import load, workloads

TUNING_DIR = Path(__file__).resolve().parent / "tuning"
SCHED_DIR = Path(__file__).resolve().parent / "schedulers"


def _device_tag() -> str:
    name = torch.cuda.get_device_name(torch.cuda.current_device())
    return re.sub(r"[^A-Za-z0-9]+", "_", name).strip("_")


def tuning_path(mech_name: str, workload: str, device_tag: Optional[str] = None) -> Path:
    return TUNING_DIR / f"{device_tag or _device_tag()}_{mech_name}_{workload}.json"


def apply(mech, workload: str) -> Optional[dict]:
    """Sets the tuned kernel and blocks per SM on `mech` when this GPU has a
    tuning record for the workload; returns the record's choice or None."""
    p = tuning_path(mech.name, workload)
    if not p.exists():
        return None
    rec = json.loads(p.read_text())
    choice = rec["choice"]
    mech.set_kernel(choice["kernel"])
    mech.set_blocks_per_sm(choice["blocks_per_sm"])
    if "queue" in choice:
        mech.set_queue_lanes(choice["queue"] == "lanes")
    return dict(choice, source=str(p.relative_to(TUNING_DIR.parent.parent)))


def candidates(mech, queue: bool = False):
    out = [{"kernel": "thread", "blocks_per_sm": b, "queue": q}
           for q in (("warps", "lanes") if queue else ("warps",)) for b in (0, 7, 6, 5, 4)]
    mech.set_kernel("warp")
    if mech.kernel() == "warp":
        out.append({"kernel": "warp", "blocks_per_sm": 0, "queue": "warps"})
    mech.set_kernel("auto")
    return out


def tune(mech_name: str, workload: str, ncells: int = 1 << 18, reps: int = 2,
         write: bool = True, verbose: bool = True) -> dict:
    mech = load(mech_name)
    wl = workloads.for_mechanism(mech, workload, ncells, seed=workloads.SEED_TRAIN + 7)
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    fix, temp, atol, rtol = D(wl.fix), D(wl.temp), D(wl.atol), D(wl.rtol)
    cf = D(wl.cfactor) if wl.cfactor is not None else None
    sun = D(wl.sun) if wl.sun is not None else None
    t0, t1 = (D(x) for x in wl.step_bounds(0))
    weights = SCHED_DIR / f"{workload}.npz"
    sched = None
    if weights.exists():
        from .scheduler import LearnedScheduler
        sched = LearnedScheduler.load(weights, mech.nvar)
    var = D(wl.var)
    hs = order = None
    if sched is not None:
        hs, order = sched.plan(var, temp, t0, cfactor=cf, sun=sun, tend=t1)

    def run(shape):
        mech.set_kernel(shape["kernel"])
        mech.set_blocks_per_sm(shape["blocks_per_sm"])
        mech.set_queue_lanes(shape["queue"] == "lanes")
        best, out = None, None
        for _ in range(reps):
            v = D(wl.var)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            if sched is not None and shape["kernel"] == "thread":
                mech.rosenbrock_chain(v, fix, temp, t0, wl.dt, 1, atol, rtol, wl.ipar, wl.rpar,
                                      cfactor=cf, sun=sun, hstart=hs, order=order)
            else:
                mech.rosenbrock(v, fix, temp, t0, t1, atol, rtol, wl.ipar, wl.rpar, cfactor=cf,
                                sun=sun, hstart=hs)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best, out = (ms, v) if best is None or ms < best else (best, out)
        return best, out

    table, ref = [], None
    for shape in candidates(mech, queue=sched is not None):
        ms, v = run(shape)
        same = True if ref is None else bool(torch.equal(v, ref))
        ref = v if ref is None else ref
        table.append(dict(shape, ms=round(ms, 2), identical=same))
        if verbose:
            print(json.dumps(table[-1]), flush=True)
    mech.set_kernel("auto")
    mech.set_blocks_per_sm(0)
    mech.set_queue_lanes(True)  # the library's default
    if not all(t["identical"] for t in table):
        raise RuntimeError("launch shapes gave different results")
    best = min(table, key=lambda t: t["ms"])
    rec = {"device": torch.cuda.get_device_name(), "mechanism": mech_name, "workload": workload,
           "sample_cells": ncells, "path": "learned plan + work queue" if sched else "plain",
           "choice": {"kernel": best["kernel"], "blocks_per_sm": best["blocks_per_sm"],
                      "queue": best["queue"]},
           "table": table}
    if write:
        TUNING_DIR.mkdir(exist_ok=True)
        tuning_path(mech_name, workload).write_text(json.dumps(rec, indent=1) + "\n")
    return rec


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--mech", default="saprc99")
    ap.add_argument("--workload", default="saprc99_uniform95")
    ap.add_argument("--ncells", type=int, default=1 << 18)
    args = ap.parse_args(argv)
    rec = tune(args.mech, args.workload, args.ncells)
    print(json.dumps({k: rec[k] for k in ("device", "mechanism", "workload", "choice")}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
