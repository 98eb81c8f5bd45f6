#!/usr/bin/env python
"""Benchmark: saprc99 cell-steps/s of the batched Rosenbrock path on B200.

One "step" is one chemistry step (600 s, Rodas3, RTOL 1e-3, ATOL 1e-2) of
every grid cell of the batch: the batched counterpart of one INTEGRATE call
per cell (int/rosenbrock.c:94-133).  The default workload is saprc99 at
2^20 cells with the config-2 input distribution (seeded synthetic cells,
kpp_b200/workloads.py), as the headline metric is quoted:
  --mode fresh  (default) every step integrates the same fresh batch from its
                initial state with the default starting step (STEPMIN = 0),
                the case a learned starting step and cost binning address;
  --mode chain  the cells' state carries over from step to step and each step
                warm-starts from the previous step's Hexit, as INTEGRATE does.

Arms
  --impl kpp_b200   (default) the CUDA path.  `value` is device-timed with
                    inputs resident in HBM; `e2e` is the same metric through
                    the public API with host buffers (pinned host -> device
                    copy of every input and device -> host copy of every
                    output inside the timed region).
  --impl reference  the reference's own CPU implementation (the KPP-generated
                    C model with the reference Rosenbrock, oracle/_ref, -O as
                    in util/Makefile_c) on all host cores, one process per
                    core (the generated code keeps its state in globals), each
                    step a bounded sample of the same workload.

Multi-GPU (torchrun): cells are independent, so each rank integrates its own
shard of 2^20 cells (weak scaling, no collective on the data path); the
timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "saprc99 cell-steps/s at 2^20 cells, learned-scheduled vs plain"
UNIT = "cell-steps/s"


# ---------------------------------------------------------------------------
# CPU baseline / reference arm (oracle libraries, separate processes)
# ---------------------------------------------------------------------------
def _cpu_worker(args):
    mech, lib_opt, sl_var, sl_fix, temp, cf, sun, t0, t1, atol, rtol, ipar, rpar = args
    sys.path.insert(0, str(REPO / "tests"))
    from oracle_lib import OracleLib
    o = OracleLib(mech, lib_opt)
    t = time.perf_counter()
    o.integrate(sl_var, sl_fix, temp, t0, t1, atol, rtol, ipar, rpar, cfactor=cf, sun=sun)
    return time.perf_counter() - t


def cpu_reference_rate(wl, ncells_sample: int, procs: int, lib_opt: str = "", pool=None):
    """cell-steps/s of the reference C path on `procs` processes, each
    integrating a contiguous slice of the first `ncells_sample` cells."""
    sub = wl.subset(ncells_sample)
    t0, t1 = sub.step_bounds(0)
    bounds = np.linspace(0, ncells_sample, procs + 1).astype(int)
    jobs = []
    for p in range(procs):
        a, b = bounds[p], bounds[p + 1]
        if b <= a:
            continue
        sl = slice(a, b)
        opt = lambda x: None if x is None else np.ascontiguousarray(x[sl])
        jobs.append((wl.mech, lib_opt, np.ascontiguousarray(sub.var[:, sl]),
                     np.ascontiguousarray(sub.fix[:, sl]), sub.temp[sl], opt(sub.cfactor),
                     opt(sub.sun), t0[sl], t1[sl], sub.atol, sub.rtol, sub.ipar, sub.rpar))
    t = time.perf_counter()
    pool.map(_cpu_worker, jobs)
    wall = time.perf_counter() - t
    return ncells_sample / wall, wall


def calibrated_sample(wl, procs, pool, target_s=12.0, lib_opt=""):
    """Pick a sample size that takes about target_s of wall time."""
    probe = max(procs * 4, 64)
    rate, wall = cpu_reference_rate(wl, probe, procs, lib_opt, pool)
    n = int(min(wl.ncells, max(probe, rate * target_s)))
    return n, rate


def host_cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# the CUDA arm
# ---------------------------------------------------------------------------
def fp64_peak(util_lib):
    import ctypes
    lib = ctypes.CDLL(str(util_lib))
    lib.kpp_b200_fp64_peak_tflops.restype = ctypes.c_double
    lib.kpp_b200_fp64_peak_tflops.argtypes = [ctypes.c_int, ctypes.c_int]
    return lib.kpp_b200_fp64_peak_tflops(0, 5), lib.kpp_b200_fp64_peak_tflops(1, 5)


def method_vector_ops(nvar: int, method: str, fixed_rates: bool) -> dict:
    """FP64 operations of the integrator outside the mechanism functions, per
    step attempt (vector updates, error norm) and per step (dF/dT)."""
    sys.path.insert(0, str(REPO / "tests"))
    from kpp_b200.controls import METHODS
    m = METHODS[method]
    # stages, nonzero A, nonzero C, nonzero gamma, nonzero M, nonzero E (Rosenbrock tableaux)
    tab = {1: (2, 1, 1, 2, 2, 2), 2: (3, 2, 3, 3, 3, 3), 3: (4, 5, 6, 4, 4, 4),
           4: (4, 3, 6, 2, 3, 1), 5: (6, 15, 15, 4, 6, 1)}[m]
    s, na, nc, ng, nm, ne = tab
    per_attempt = 2 * nvar * (na + nc + ng + nm + ne) + 6 * nvar + 2 * s + 8
    per_step = 3 * nvar
    return {"per_attempt": per_attempt, "per_step": per_step}


def run_cuda_arm(args, rank, world, local_rank):
    import torch
    from kpp_b200 import load, workloads
    from kpp_b200.build import LIB

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    mech = load(args.mech)
    mech.set_kernel(args.kernel)
    kernel = mech.kernel()
    wl = workloads.for_mechanism(mech, args.workload, args.ncells, seed=workloads.SEED_EVAL + rank)
    n = wl.ncells
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    var = D(wl.var)
    fix, temp = D(wl.fix), D(wl.temp)
    cf = D(wl.cfactor) if wl.cfactor is not None else None
    sun = D(wl.sun) if wl.sun is not None else None
    atol, rtol = D(wl.atol), D(wl.rtol)
    total = args.warmup + args.steps
    t_bounds = [(D(wl.step_bounds(k)[0]), D(wl.step_bounds(k)[1])) for k in range(total)]
    hstart = torch.zeros(n, dtype=torch.float64, device=dev)
    out = None
    stream = torch.cuda.current_stream(dev)

    fresh = args.mode == "fresh"
    var0 = var.clone() if fresh else None

    def step(k):
        nonlocal out, hstart
        if fresh:
            var.copy_(var0)  # the same fresh batch every step
            out = mech.rosenbrock(var, fix, temp, t_bounds[0][0], t_bounds[0][1], atol, rtol,
                                  wl.ipar, wl.rpar, cfactor=cf, sun=sun, out=out)
            return
        out = mech.rosenbrock(var, fix, temp, t_bounds[k][0], t_bounds[k][1], atol, rtol,
                              wl.ipar, wl.rpar, cfactor=cf, sun=sun, hstart=hstart, out=out)
        hstart = out.rstatus[1].clone()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()

    # state at the start of the timed steps; the end-to-end run replays the
    # same steps from it
    snap_var = (var0 if fresh else var).cpu().numpy().copy()
    snap_hs = hstart.cpu().numpy().copy()

    # ---- device-timed region: inputs resident in HBM (larger than L2)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for k in range(args.warmup, total):
            step(k)
            stats.append(out.istatus.sum(dim=1))  # device-side reduction, no sync
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    ierr = out.ierr.cpu().numpy()
    ist_sum = torch.stack(stats).sum(dim=0).cpu().numpy().astype(np.int64)
    ms_max = ms
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * n * args.steps / (ms_max / 1e3)

    # ---- algorithmic FP64 work of the timed steps (exact counts from ISTATUS)
    hdr = (REPO / "kpp_b200" / "_gen" / f"{args.mech}.cuh")
    opsd = {}
    if hdr.exists():
        for line in hdr.read_text().splitlines():
            if line.startswith("#define KPP_OPS_"):
                _, k, v = line.split()
                opsd[k[8:].lower()] = int(v)
    nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng = ist_sum.tolist()
    fixed_rates = sun is not None
    vec = method_vector_ops(mech.nvar, "rodas3", fixed_rates)
    fun_evals = nfun - (njac if fixed_rates else 0)   # dF/dT Fun elided for fixed rates
    flops = (fun_evals * opsd.get("fun", 0) + ndec * (opsd.get("jac", 0) + opsd.get("decomp", 0))
             + nsol * opsd.get("solve", 0) + nstp * vec["per_attempt"] + njac * vec["per_step"])
    achieved_tflops = flops / (ms / 1e3) / 1e12
    peak_fma, peak_muladd = fp64_peak(LIB / "libkpp_b200_util.so")

    # ---- end to end through the public API with host buffers: the same timed
    # steps, from the same state, through kpp_b200_rosenbrock_host (pinned host
    # arrays in, results back in host memory every step)
    e2e = None
    if args.e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        h_var, h_fix, h_temp = pin(snap_var), pin(wl.fix), pin(wl.temp)
        h_cf = pin(wl.cfactor) if wl.cfactor is not None else None
        h_sun = pin(wl.sun) if wl.sun is not None else None
        h_atol, h_rtol = pin(wl.atol), pin(wl.rtol)
        h_t = [(pin(wl.step_bounds(k)[0]), pin(wl.step_bounds(k)[1])) for k in range(total)]
        h_hs = pin(snap_hs)
        res = None

        h_var0 = h_var.clone() if fresh else None

        def e2e_step(k):
            nonlocal res
            if fresh:
                h_var.copy_(h_var0)  # the host model hands in the same fresh cells
                res = mech.rosenbrock_host(h_var, h_fix, h_temp, h_t[0][0], h_t[0][1], h_atol,
                                           h_rtol, wl.ipar, wl.rpar, cfactor=h_cf, sun=h_sun,
                                           out=res)
                return
            res = mech.rosenbrock_host(h_var, h_fix, h_temp, h_t[k][0], h_t[k][1], h_atol, h_rtol,
                                       wl.ipar, wl.rpar, cfactor=h_cf, sun=h_sun, hstart=h_hs,
                                       out=res)
            h_hs.copy_(res.rstatus[1])  # the host model's warm start for its next call

        keep_var, keep_hs = h_var.clone(), h_hs.clone()
        e2e_step(args.warmup)  # warm the pipeline, then replay the timed steps
        h_var.copy_(keep_var)
        h_hs.copy_(keep_hs)
        torch.cuda.synchronize()
        barrier()
        t_start = time.perf_counter()
        for k in range(args.warmup, total):
            e2e_step(k)
        ems = (time.perf_counter() - t_start) * 1e3
        barrier()
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        nb = lambda x: 0 if x is None else x.numel() * x.element_size()
        h2d = sum(nb(x) for x in (h_var, h_fix, h_temp, h_cf, h_sun, h_t[0][0], h_t[0][1],
                                  None if fresh else h_hs))
        d2h = nb(h_var) + nb(res.istatus) + nb(res.rstatus) + nb(res.ierr)
        same = bool(np.array_equal(h_var.numpy(), var.cpu().numpy()))
        e2e = {"value": world * n * args.steps / (ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": ems / args.steps, "api": "kpp_b200_rosenbrock_host (pinned host "
               "arrays, chunked copies overlapped with the integration, synchronous)",
               "matches_device_run": same}

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.mech} {args.workload} ({args.mode}) plain Rodas3, {n} cells "
                               f"per GPU, 600 s chemistry step, RTOL 1e-3 ATOL 1e-2",
                   "mode": args.mode,
                   "cells_per_gpu": n, "chemistry_step_s": wl.dt, "method": "rodas3",
                   "scheduler": "plain", "parallelism": f"cell shards x{world}",
                   "kernel": {"thread": "thread per cell", "warp": "warp per cell"}[kernel],
                   "l2": "inputs larger than L2 (VAR alone %d MB)" % (wl.var.nbytes >> 20)},
        "impl": "kpp_b200",
        "gpu_launches": args.steps * (2 if kernel == "warp" else 1),
        "stats": {"internal_steps_per_cell_step": nstp / (n * args.steps),
                  "rejected_per_cell_step": nrej / (n * args.steps),
                  "ierr_ok_fraction": float((ierr == 1).mean()),
                  "istatus_sum": dict(zip(["nfun", "njac", "nstp", "nacc", "nrej", "ndec", "nsol",
                                           "nsng"], map(int, ist_sum)))},
        "roofline": {"bound": "fp64", "achieved": achieved_tflops, "peak": peak_fma,
                     "unit": "TFLOP/s", "frac": achieved_tflops / peak_fma if peak_fma > 0 else None,
                     "traffic": None,
                     "peak_source": "measured on this GPU by the DFMA throughput kernel "
                                    "(kpp_b200/csrc/kpp_util.cu); MEASURED_PEAKS.json has no FP64 figure",
                     "peak_mul_add_tflops": peak_muladd,
                     "flops_per_cell_step": flops / (n * args.steps)},
        "clocks": clk.summary(),
        "e2e": e2e,
    }
    return result, wl


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--mode", choices=["fresh", "chain"], default="fresh")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["kpp_b200", "reference"], default="kpp_b200")
    ap.add_argument("--mech", default="saprc99")
    ap.add_argument("--workload", default="saprc99_uniform95")
    ap.add_argument("--ncells", type=int, default=1 << 20)
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--kernel", choices=["auto", "thread", "warp"], default="auto")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    procs = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return 0
        ctx = mp.get_context("spawn")
        from kpp_b200 import load, workloads
        mech = load(args.mech)
        wl = workloads.for_mechanism(mech, args.workload, args.ncells, seed=workloads.SEED_EVAL)
        with ctx.Pool(procs) as pool:
            n_sample, _ = calibrated_sample(wl, procs, pool, target_s=min(args.cpu_seconds, 20.0))
            for _ in range(args.warmup and 1):
                cpu_reference_rate(wl, max(procs * 4, 64), procs, "", pool)
            rates, walls = [], []
            for _ in range(args.steps):
                r, w = cpu_reference_rate(wl, n_sample, procs, "", pool)
                rates.append(r)
                walls.append(w)
        v = statistics.median(rates)
        line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(walls),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": f"{args.mech} {args.workload} plain Rodas3, 600 s chemistry "
                                       f"steps, RTOL 1e-3 ATOL 1e-2; each step a sample of "
                                       f"{n_sample} of the {args.ncells} cells"},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": "reference",
                                 "sample": f"{n_sample} cells x 1 chemistry step per timed step, "
                                           f"{procs} processes, KPP-generated C + int/rosenbrock.c "
                                           f"(gcc -O), host CPU {host_cpu_model()}"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "gpu_launches": 0}
        print(json.dumps(line), flush=True)
        return 0

    # spawn the CPU pool before the first CUDA call
    ctx = mp.get_context("spawn")
    pool = ctx.Pool(procs) if (args.cpu_baseline and rank == 0 and world == 1) else None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    result, wl = run_cuda_arm(args, rank, world, local_rank)
    if pool is not None:
        n_sample, _ = calibrated_sample(wl, procs, pool, target_s=args.cpu_seconds)
        rate, wall = cpu_reference_rate(wl, n_sample, procs, "", pool)
        pool.close()
        result["cpu_baseline"] = {
            "value": rate, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{n_sample} cells x 1 chemistry step of the same workload, {procs} processes "
                      f"(reference KPP-generated C + int/rosenbrock.c, gcc -O), {wall:.1f} s wall, "
                      f"host CPU {host_cpu_model()}"}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
