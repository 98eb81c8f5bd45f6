"""Train the learned scheduler of a mechanism on the GPU.

  python -m kpp_b200.train_scheduler --mech saprc99 --workload saprc99_uniform95 \
      --ncells 4194304 --out kpp_b200/schedulers/saprc99_uniform95.npz

Logs (features, best Hstart, step count) tuples from the plain GPU integrator
over `ncells` cells drawn with the training seed (workloads.SEED_TRAIN, not
the evaluation seed), fits the network with the library's kernels and writes
the weights with their scaling.  Prints one JSON line with the fit summary.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import torch

from . import load, workloads
from . import scheduler as S

DEFAULT_DIR = Path(__file__).resolve().parent / "schedulers"


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--mech", default="saprc99")
    ap.add_argument("--workload", default="saprc99_uniform95")
    ap.add_argument("--ncells", type=int, default=1 << 22)
    ap.add_argument("--epochs", type=int, default=24)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=workloads.SEED_TRAIN)
    ap.add_argument("--out", type=Path, default=None)
    args = ap.parse_args(argv)
    out = args.out or DEFAULT_DIR / f"{args.workload}.npz"

    torch.cuda.set_device(0)
    mech = load(args.mech)
    t0 = time.time()
    wl = workloads.for_mechanism(mech, args.workload, args.ncells, seed=args.seed)
    print(f"workload {wl.name}: {wl.ncells} cells (seed {args.seed}), "
          f"{time.time() - t0:.1f} s", flush=True)
    t1 = time.time()
    nstp, ok = S.log_tuples(mech, wl)
    log_s = time.time() - t1
    sch = S.train(wl, nstp, ok, epochs=args.epochs, batch=args.batch, lr=args.lr,
                  seed=args.seed)
    out.parent.mkdir(parents=True, exist_ok=True)
    sch.save(out)
    best = nstp.min(axis=0)
    summary = dict(sch.meta)
    summary.update({"out": str(out), "tuple_logging_seconds": round(log_s, 1),
                    "mean_nstp_default_hstart": float(nstp[0].mean()),
                    "mean_nstp_best_candidate": float(best.mean()),
                    "failed_cells": int((~ok).sum())})
    print(json.dumps(summary), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
