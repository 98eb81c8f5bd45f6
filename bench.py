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
                warm-starts from the previous step's Hexit, as INTEGRATE does;
  --mode diurnal  24 chained steps of cells of uneven stiffness, one launch per
                step against one persistent work-queue launch;
  --mode sdirk / --mode rk  the same fresh batch with the reference's other C
                integrators (int/sdirk.c, --sdirk-method; int/runge_kutta.c,
                --rk-method), their reference arms timing the reference's own
                SDIRK / RungeKutta.

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

METRIC = "saprc99 cell-steps/s at 2^20 cells, learned-scheduled vs plain, same accuracy"
UNIT = "cell-steps/s"
# DRAM traffic per internal step of each Rosenbrock kernel at full residency
# (ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch over fresh
# saprc99 cells):
#   thread per cell: 2^17 cells, every thread slot of the GPU busy: 990.0 +
#     311.4 GB over 6,480,123 internal steps
#     (profiles/rosenbrock_kernel_thread_saprc99_2p17_traffic.md): the
#     per-cell work set (LU factors, stage vectors) streams through L2 to HBM;
#   warp per cell: 2048 cells (every SM's 12 cells busy, then a tail):
#     1.75 MB read, 0 written over 101,110 internal steps
#     (profiles/kernel_coop_saprc99_2048_fresh.md): the work set stays in
#     shared memory; what remains is the cells' inputs and outputs.
DRAM_BYTES_PER_INTERNAL_STEP = {"thread": (989962676736 + 311353660160) / 6480123,
                                "warp": 1750528 / 101110}
TRAFFIC_SOURCE = {
    "thread": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one rosenbrock_kernel "
              "launch over 2^17 fresh cells at full residency (profiles/), per internal step, "
              "times this launch's internal steps",
    "warp": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one warp-per-cell kernel "
            "launch over 2048 fresh cells, every SM's cells busy (profiles/), per internal "
            "step, times this launch's internal steps"}
# Compulsory bytes per cell-step: VAR in and out, FIX, TEMP, CFACTOR, SUN,
# TSTART, TEND, Hstart in; ISTATUS, RSTATUS, IERR out (saprc99: 74 + 74 + 5 +
# 6 doubles, 9 ints, 2 doubles).
ALGO_BYTES_PER_CELL_STEP = (74 + 74 + 5 + 6) * 8 + 9 * 4 + 2 * 8
# How the committed scheduler weights were made (python -m kpp_b200.train_scheduler
# on one B200): tuples logged from the plain GPU integrator, seed 20261204.
TRAINING_SUMMARY = {
    "saprc99_uniform95": {
        "tuples": 4194304, "candidates_hstart": "1e-6 .. 1e-2 s, half decades",
        "tuple_logging_s": 247.7, "epochs": 24, "batch": 8192, "train_s": 19.6,
        "heldout_r2_log10_hstart": 0.918, "heldout_r2_ln_nstp": 0.974,
        "mean_nstp_default_hstart": 49.42, "mean_nstp_best_candidate": 46.03},
}


# ---------------------------------------------------------------------------
# CPU baseline / reference arm (oracle libraries, separate processes)
# ---------------------------------------------------------------------------
def _cpu_worker(args):
    mech, lib_opt, sl_var, sl_fix, temp, cf, sun, t0, t1, atol, rtol, ipar, rpar, integ = args
    sys.path.insert(0, str(REPO / "tests"))
    # the reference integrators print their error messages with printf: keep
    # them off this pool process's stdout (the bench prints one JSON line)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    os.close(null)
    if integ is not None and integ[0] == "adj":
        from oracle_lib import AdjOracle
        o = AdjOracle(mech, lib_opt)
        lam = np.random.default_rng(7).standard_normal((integ[3] * o.nvar, sl_var.shape[1]))
        t = time.perf_counter()
        o.integrate(sl_var, sl_fix, temp, t0, t1, atol, rtol, lam, integ[1], integ[2], integ[4],
                    cfactor=cf, sun=sun)
        return time.perf_counter() - t
    if integ is not None:
        from oracle_lib import RkOracle, SdirkOracle
        o = (SdirkOracle if integ[0] == "sdirk" else RkOracle)(mech, lib_opt)
        t = time.perf_counter()
        o.integrate(sl_var, sl_fix, temp, t0, t1, atol, rtol, integ[1], integ[2],
                    cfactor=cf, sun=sun)
        return time.perf_counter() - t
    from oracle_lib import OracleLib
    o = OracleLib(mech, lib_opt)
    t = time.perf_counter()
    o.integrate(sl_var, sl_fix, temp, t0, t1, atol, rtol, ipar, rpar, cfactor=cf, sun=sun)
    return time.perf_counter() - t


def cpu_reference_rate(wl, ncells_sample: int, procs: int, lib_opt: str = "", pool=None,
                       integ=None):
    """cell-steps/s of the reference C path on `procs` processes, each
    integrating a contiguous slice of the first `ncells_sample` cells; with
    `integ` = (kind, ICNTRL, RCNTRL) the reference's SDIRK ("sdirk") or
    Runge-Kutta ("rk") integrator instead of its Rosenbrock."""
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
        fix = sub.fix if sub.fix.shape[0] else np.zeros((1, ncells_sample))  # C pads NFIX
        jobs.append((wl.mech, lib_opt, np.ascontiguousarray(sub.var[:, sl]),
                     np.ascontiguousarray(fix[:, sl]), sub.temp[sl], opt(sub.cfactor),
                     opt(sub.sun), t0[sl], t1[sl], sub.atol, sub.rtol, sub.ipar, sub.rpar, integ))
    t = time.perf_counter()
    pool.map(_cpu_worker, jobs)
    wall = time.perf_counter() - t
    return ncells_sample / wall, wall


def calibrated_sample(wl, procs, pool, target_s=12.0, lib_opt="", integ=None):
    """Pick a sample size that takes about target_s of wall time."""
    probe = max(procs * 4, 64)
    rate, wall = cpu_reference_rate(wl, probe, procs, lib_opt, pool, integ)
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
# multi-GPU plumbing: independent shards, device timing reduced by max
# ---------------------------------------------------------------------------
def shard_seed(rank: int) -> int:
    """Each rank integrates its own shard of cells, drawn with the evaluation
    seed + rank (no exchange of cell data between ranks)."""
    from kpp_b200 import workloads
    return workloads.SEED_EVAL + rank


def reduce_max(value: float, device) -> float:
    """The largest value over all ranks (the job ends with its slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank: int, world: int, steps: int, ms_max: float) -> float:
    """cell-steps/s of the whole job: every rank's cells over the slowest rank's time."""
    return world * cells_per_rank * steps / (ms_max / 1e3)


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
            self._first.set()
            self._stop.wait(0.2)

    def __enter__(self):
        self._first = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        # the first query (thread start, process spawn) before the timed
        # region opens, so that short steps do not carry it
        self._first.wait(timeout=5.0)
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


def _tight_worker(args):
    mech, var, fix, temp, cf, sun, t0, t1, ipar, rpar = args
    sys.path.insert(0, str(REPO / "tests"))
    from oracle_lib import OracleLib
    o = OracleLib(mech)
    v, _, _, ierr = o.integrate(var, fix, temp, t0, t1, np.array([TIGHT_ATOL]),
                                np.array([TIGHT_RTOL]), ipar, rpar, cfactor=cf, sun=sun,
                                which="or")
    return v, ierr


TIGHT_RTOL, TIGHT_ATOL = 1e-10, 1e-8


def tight_reference(wl, cells, pool):
    """FP64 Rodas4 solution at RTOL 1e-10 (ATOL 1e-8 molec/cm3, at most 10^6
    steps) of the given
    cells from their initial state over the first chemistry step, by the CPU
    restatement of the reference Rosenbrock (oracle/ros_oracle.c)."""
    from kpp_b200.controls import make_controls
    # up to 10^6 steps: some MCM cells need more than the default 100000 at
    # RTOL 1e-10 (step sizes near 1e-3 s over a 300 s step)
    ipar, rpar = make_controls(method="rodas4", scalar_tol=True, max_steps=1_000_000)
    t0, t1 = wl.step_bounds(0)
    parts = np.array_split(cells, min(len(cells), os.cpu_count() or 1))
    opt = lambda x, c: None if x is None else np.ascontiguousarray(x[c])
    jobs = [(wl.mech, np.ascontiguousarray(wl.var[:, c]), np.ascontiguousarray(wl.fix[:, c]),
             wl.temp[c], opt(wl.cfactor, c), opt(wl.sun, c), t0[c], t1[c], ipar, rpar)
            for c in parts if len(c)]
    res = pool.map(_tight_worker, jobs)
    return np.concatenate([r[0] for r in res], axis=1), np.concatenate([r[1] for r in res])


def tight_gpu(mech, wl, cells, dev, ncalls: int = 1):
    """The same FP64 Rodas4 RTOL 1e-10 solution as tight_reference, for the
    given cells, by the library's own integrator (whose parity with the
    reference the tests establish); with ncalls > 1, over the driver loop of
    ncalls chemistry steps (kpp_b200_rosenbrock_chain).  Returns (var, ierr,
    ms)."""
    import torch
    from kpp_b200.controls import make_controls
    ipar, rpar = make_controls(method="rodas4", scalar_tol=True, max_steps=1_000_000)
    D = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    t0, t1 = wl.step_bounds(0)
    var = D(wl.var[:, cells])
    args = dict(cfactor=None if wl.cfactor is None else D(wl.cfactor[cells]),
                sun=None if wl.sun is None else D(wl.sun[cells]))
    tol = (D(np.array([TIGHT_ATOL])), D(np.array([TIGHT_RTOL])))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    if ncalls == 1:
        r = mech.rosenbrock(var, D(wl.fix[:, cells]), D(wl.temp[cells]), D(t0[cells]),
                            D(t1[cells]), *tol, ipar, rpar, **args)
    else:
        r = mech.rosenbrock_chain(var, D(wl.fix[:, cells]), D(wl.temp[cells]),
                                  D(wl.tstart[cells]), wl.dt, ncalls, *tol, ipar, rpar, **args)
    e1.record()
    torch.cuda.synchronize()
    return var.cpu().numpy(), r.ierr.cpu().numpy(), e0.elapsed_time(e1)


def accuracy_block(mech, wl, got, ncells, ncalls, dev, ncheck):
    """accuracy() of a result `got` [NVAR, n] over `ncheck` cells evenly
    spaced over the batch, against tight_gpu's solution of the same cells."""
    cells = np.unique(np.linspace(0, ncells - 1, min(ncheck, ncells)).astype(np.int64))
    ref, ref_ierr, tight_ms = tight_gpu(mech, wl, cells, dev, ncalls)
    ok = ref_ierr == 1
    out = accuracy(got[:, cells[ok]], ref[:, ok], float(wl.atol[0]), float(wl.rtol[0])) \
        if ok.any() else None
    return {"result": out,
            "oracle": f"FP64 Rodas4, RTOL {TIGHT_RTOL:g}, ATOL {TIGHT_ATOL:g}, at most 10^6 "
                      f"steps per call, {ncalls} chained call(s), on the GPU "
                      f"({tight_ms / 1e3:.1f} s); cells evenly spaced over the batch",
            "oracle_cells_ok": int(ok.sum()), "oracle_cells": int(ok.size)}


def accuracy(got: np.ndarray, ref: np.ndarray, atol: float, rtol: float) -> dict:
    """Error of an RTOL 1e-3 solution against the tight one: the largest
    relative error over species above 1e3 ATOL (where the relative tolerance
    governs the solve), and the largest per-cell error in the integrator's own
    norm, sqrt(mean(((y - ref) / (ATOL + RTOL |ref|))^2))."""
    mask = np.abs(ref) > 1e3 * atol
    rel = np.abs(got - ref)[mask] / np.abs(ref)[mask]
    norm = np.sqrt((((got - ref) / (atol + rtol * np.abs(ref))) ** 2).mean(axis=0))
    return {"max_rel_err_above_1e3_atol": float(rel.max()) if rel.size else None,
            "median_rel_err_above_1e3_atol": float(np.median(rel)) if rel.size else None,
            "max_cell_error_norm": float(norm.max()), "cells": int(ref.shape[1])}


def run_cuda_arm(args, rank, world, local_rank, pool=None):
    import torch
    from kpp_b200 import load, workloads
    from kpp_b200.build import LIB

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    mech = load(args.mech)
    mech.set_kernel(args.kernel)
    shape = None
    if args.kernel == "auto":
        from kpp_b200 import autotune
        shape = autotune.apply(mech, args.workload)  # tuned on this GPU, if recorded
    if args.queue != "tuned":
        mech.set_queue_lanes(args.queue == "lanes")  # an explicit choice wins
    queue = "lanes" if mech.queue_lanes() else "warps"
    wl = workloads.for_mechanism(mech, args.workload, args.ncells, seed=shard_seed(rank))
    n = wl.ncells
    # the kernel choice of the headline arms: the tuning record's, else the
    # command line's (auto: the library's automatic choice)
    arm_kernel = shape["kernel"] if shape else args.kernel
    mech.set_kernel("warp")
    has_warp = mech.kernel() == "warp" and wl.sun is not None
    mech.set_kernel(arm_kernel)
    kernel = ("warp" if has_warp else "thread") if arm_kernel == "auto" else arm_kernel
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    var = D(wl.var)
    fix, temp = D(wl.fix), D(wl.temp)
    cf = D(wl.cfactor) if wl.cfactor is not None else None
    sun = D(wl.sun) if wl.sun is not None else None
    atol, rtol = D(wl.atol), D(wl.rtol)
    total = args.warmup + args.steps
    t_bounds = [(D(wl.step_bounds(k)[0]), D(wl.step_bounds(k)[1])) for k in range(total)]
    stream = torch.cuda.current_stream(dev)
    fresh = args.mode == "fresh"
    var0 = var.clone()

    sched, sched_note = None, None
    if args.scheduler == "learned":
        from kpp_b200.scheduler import LearnedScheduler
        wpath = Path(args.weights) if args.weights else (
            REPO / "kpp_b200" / "schedulers" / f"{args.workload}.npz")
        if wpath.exists():
            sched = LearnedScheduler.load(wpath, mech.nvar)
        else:
            sched_note = f"no trained scheduler at {wpath}: plain only"

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(ms):
        return ms if world == 1 else reduce_max(ms, dev)

    class Arm:
        """One way of running the steps: plain (grid-stride kernel, Hstart =
        STEPMIN), learned (plan, then the work-queue kernel in cost order
        with the planned Hstart) or, with `fixed` = (Hstart, order) tensors,
        the work-queue kernel with a given Hstart and order (the ceiling arm:
        each cell's best starting step among the training candidates, queued
        by its true step count)."""

        def __init__(self, learned, fixed=None, kernel=None):
            self.learned = learned
            self.fixed = fixed
            self.kernel = kernel  # a kernel choice for this arm's launches, else the tuned one
            self.out = None
            self.hs = torch.zeros(n, dtype=torch.float64, device=dev)
            self.hs_plan = torch.empty(n, dtype=torch.float64, device=dev)
            self.order = torch.empty(n, dtype=torch.int32, device=dev)
            # events around the integration launch of each timed step (on the
            # stream it runs on): the dominant kernel's own duration
            self.kernel_events = {}

        def step(self, k):
            kk = 0 if fresh else k
            if fresh:
                var.copy_(var0)  # the same fresh batch every step
            t0, t1 = t_bounds[kk]
            warm = None if fresh else self.hs
            ev = self.kernel_events[k] if self.kernel_events else None
            if self.fixed is not None:
                if ev:
                    ev[0].record(stream)
                self.out = mech.rosenbrock_chain(
                    var, fix, temp, t0, wl.dt, 1, atol, rtol, wl.ipar, wl.rpar, cfactor=cf,
                    sun=sun, hstart=self.fixed[0], order=self.fixed[1], out=self.out)
            elif not self.learned:
                if self.kernel is not None:
                    mech.set_kernel(self.kernel)
                if ev:
                    ev[0].record(stream)
                self.out = mech.rosenbrock(var, fix, temp, t0, t1, atol, rtol, wl.ipar, wl.rpar,
                                           cfactor=cf, sun=sun, hstart=warm, out=self.out)
                if self.kernel is not None:
                    mech.set_kernel(arm_kernel)
            else:
                sched.plan(var, temp, t0, cfactor=cf, sun=sun, tend=t1, hstart=self.hs_plan,
                           order=self.order)
                if ev:
                    ev[0].record(stream)
                self.out = mech.rosenbrock_chain(
                    var, fix, temp, t0, wl.dt, 1, atol, rtol, wl.ipar, wl.rpar, cfactor=cf,
                    sun=sun, hstart=self.hs_plan if fresh else warm, order=self.order,
                    out=self.out)
            if ev:
                ev[1].record(stream)
            if not fresh:
                self.hs = self.out.rstatus[1].clone()

        def run(self):
            """Warm-up steps, then the timed steps; returns ms and ISTATUS sums."""
            var.copy_(var0)
            self.hs.zero_()
            for k in range(args.warmup):
                self.step(k)
            torch.cuda.synchronize()
            self.snap_var = var.cpu().numpy() if not fresh else None
            self.snap_hs = self.hs.cpu().numpy().copy()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            self.kernel_events = {k: (torch.cuda.Event(enable_timing=True),
                                      torch.cuda.Event(enable_timing=True))
                                  for k in range(args.warmup, total)}
            stats = []
            barrier()
            torch.cuda.synchronize()
            with ClockSampler(local_rank) as clk:
                ev0.record(stream)
                for k in range(args.warmup, total):
                    self.step(k)
                    stats.append(self.out.istatus.sum(dim=1))  # device reduction, no sync
                ev1.record(stream)
                torch.cuda.synchronize()
            barrier()
            self.ms = max_over_ranks(ev0.elapsed_time(ev1))
            self.kernel_ms = sum(a.elapsed_time(b) for a, b in self.kernel_events.values())
            self.kernel_events = {}
            self.clocks = clk.summary()
            self.ierr = self.out.ierr.cpu().numpy()
            self.var_out = var.cpu().numpy()
            self.ist = torch.stack(stats).sum(dim=0).cpu().numpy().astype(np.int64)
            self.value = whole_job_rate(n, world, args.steps, self.ms)
            return self

        def summary(self):
            nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng = self.ist.tolist()
            return {"value": self.value, "unit": UNIT, "ms_per_step": self.ms / args.steps,
                    "internal_steps_per_cell_step": nstp / (n * args.steps),
                    "rejected_step_rate": nrej / max(nstp, 1),
                    "ierr_ok_fraction": float((self.ierr == 1).mean()),
                    "clocks": self.clocks,
                    "istatus_sum": dict(zip(["nfun", "njac", "nstp", "nacc", "nrej", "ndec",
                                             "nsol", "nsng"], map(int, self.ist)))}

    # the plain form: one launch per step with the library's automatic kernel
    # choice (the warp-per-cell kernel where the mechanism has it), and, for
    # comparison, the thread-per-cell kernel's plain launch
    plain_kernel = ("warp" if has_warp else "thread") if args.kernel == "auto" else args.kernel
    plain = Arm(False, kernel=args.kernel).run()
    plain_thread = (Arm(False, kernel="thread").run()
                    if fresh and plain_kernel != "thread" and args.plain_thread else None)
    # the work queue alone: the plain controls (Hstart = STEPMIN) and cells in
    # batch order, so its gain over plain is the queue's, none of it learned
    queued = (Arm(False, fixed=(torch.zeros(n, dtype=torch.float64, device=dev),
                                torch.arange(n, dtype=torch.int32, device=dev))).run()
              if fresh and args.queue_arm else None)
    learned = Arm(True).run() if sched is not None else None
    head = learned if learned is not None else plain
    # the ceiling of a starting step plus cost order on this workload: every
    # cell integrated once per training candidate Hstart (the plain
    # integrator), then timed with its best candidate, queued by the step
    # count that candidate took
    ceiling, ceiling_info = None, None
    if args.ceiling and fresh and learned is not None:
        from kpp_b200 import scheduler as _sch
        t_c = time.perf_counter()
        nstp_c, ok_c = _sch.log_tuples(mech, wl, verbose=False)
        best = np.argmin(nstp_c, axis=0)
        cols = np.arange(n)
        hs_best = np.asarray(_sch.CANDIDATES)[best]
        cost = nstp_c[best, cols]
        order_best = np.argsort(-cost, kind="stable").astype(np.int32)
        ceiling = Arm(False, fixed=(D(hs_best), D(order_best))).run()
        ceiling_info = {
            "what": "each cell's best Hstart among the 9 training candidates (1e-6 .. 1e-2 s, "
                    "half decades), queue sorted by the step count it took (decreasing)",
            "candidates_s": list(_sch.CANDIDATES),
            "mean_nstp_default_hstart": float(plain.ist[2] / (n * args.steps)),
            "mean_nstp_best_candidate": float(cost.mean()),
            "tuple_logging_s": time.perf_counter() - t_c,
            "ierr_identical_to_plain": bool(np.array_equal(ceiling.ierr, plain.ierr))}

    from kpp_b200.controls import METHODS
    method_name = {v: k for k, v in METHODS.items()}[wl.ipar[3]]
    method_title = {"ros2": "Ros2", "ros3": "Ros3", "ros4": "Ros4", "rodas3": "Rodas3",
                    "rodas4": "Rodas4"}[method_name]
    # ---- algorithmic FP64 work of the headline arm's timed steps (ISTATUS counts)
    hdr = (REPO / "kpp_b200" / "_gen" / f"{args.mech}.cuh")
    opsd = {}
    if hdr.exists():
        for line in hdr.read_text().splitlines():
            if line.startswith("#define KPP_OPS_"):
                _, k, v = line.split()
                opsd[k[8:].lower()] = int(v)
    nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng = head.ist.tolist()
    fixed_rates = sun is not None
    vec = method_vector_ops(mech.nvar, method_name, fixed_rates)
    fun_evals = nfun - (njac if fixed_rates else 0)   # dF/dT Fun elided for fixed rates
    flops = (fun_evals * opsd.get("fun", 0) + ndec * (opsd.get("jac", 0) + opsd.get("decomp", 0))
             + nsol * opsd.get("solve", 0) + nstp * vec["per_attempt"] + njac * vec["per_step"])
    # the dominant kernel's launches only (the scheduling pass excluded)
    achieved_tflops = flops / (head.kernel_ms / 1e3) / 1e12
    traffic_per_launch = DRAM_BYTES_PER_INTERNAL_STEP[kernel] * nstp / args.steps
    peak_fma, peak_muladd = fp64_peak(LIB / "libkpp_b200_util.so")

    # ---- end to end through the public API with host buffers (pinned host
    # arrays in, every output back in host memory, each step)
    e2e = None
    if args.e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        h_var0 = pin(wl.var if fresh else head.snap_var)
        h_var = h_var0.clone()
        h_fix, h_temp = pin(wl.fix), pin(wl.temp)
        h_cf = pin(wl.cfactor) if wl.cfactor is not None else None
        h_sun = pin(wl.sun) if wl.sun is not None else None
        h_atol, h_rtol = pin(wl.atol), pin(wl.rtol)
        h_t = [(pin(wl.step_bounds(k)[0]), pin(wl.step_bounds(k)[1])) for k in range(total)]
        h_hs = pin(head.snap_hs)
        nb = lambda x: 0 if x is None else x.numel() * x.element_size()
        if learned is not None:
            # the learned scheduler through its Python API: copy in, plan,
            # integrate in cost order, copy out
            d_in = {}
            res = {"ist": torch.empty(8, n, dtype=torch.int32).pin_memory(),
                   "rst": torch.empty(2, n, dtype=torch.float64).pin_memory(),
                   "ierr": torch.empty(n, dtype=torch.int32).pin_memory()}
            hs_d = torch.empty(n, dtype=torch.float64, device=dev)
            order_d = torch.empty(n, dtype=torch.int32, device=dev)
            out_box = [None]

            def e2e_step(k):
                kk = 0 if fresh else k
                if fresh:
                    h_var.copy_(h_var0)
                for nm, h in (("var", h_var), ("fix", h_fix), ("temp", h_temp), ("cf", h_cf),
                              ("sun", h_sun), ("atol", h_atol), ("rtol", h_rtol),
                              ("t0", h_t[kk][0]), ("t1", h_t[kk][1]),
                              ("hs", None if fresh else h_hs)):
                    if h is not None:
                        if nm not in d_in:
                            d_in[nm] = torch.empty_like(h, device=dev)
                        d_in[nm].copy_(h, non_blocking=True)
                sched.plan(d_in["var"], d_in["temp"], d_in["t0"], cfactor=d_in.get("cf"),
                           sun=d_in.get("sun"), tend=d_in["t1"], hstart=hs_d, order=order_d)
                out_box[0] = o = mech.rosenbrock_chain(
                    d_in["var"], d_in["fix"], d_in["temp"], d_in["t0"], wl.dt, 1, d_in["atol"],
                    d_in["rtol"], wl.ipar, wl.rpar, cfactor=d_in.get("cf"), sun=d_in.get("sun"),
                    hstart=hs_d if fresh else d_in["hs"], order=order_d, out=out_box[0])
                h_var.copy_(d_in["var"], non_blocking=True)
                res["ist"].copy_(o.istatus, non_blocking=True)
                res["rst"].copy_(o.rstatus, non_blocking=True)
                res["ierr"].copy_(o.ierr, non_blocking=True)
                torch.cuda.current_stream(dev).synchronize()
                if not fresh:
                    h_hs.copy_(res["rst"][1])

            h2d = sum(nb(x) for x in (h_var, h_fix, h_temp, h_cf, h_sun, h_atol, h_rtol,
                                      h_t[0][0], h_t[0][1], None if fresh else h_hs))
            d2h = nb(h_var) + nb(res["ist"]) + nb(res["rst"]) + nb(res["ierr"])
            api = ("kpp_b200.scheduler.LearnedScheduler.plan + Mechanism.rosenbrock_chain "
                   "(kpp_sched_plan + kpp_b200_rosenbrock_chain), pinned host arrays copied in "
                   "and out every step")
        else:
            res_box = [None]

            def e2e_step(k):
                kk = 0 if fresh else k
                if fresh:
                    h_var.copy_(h_var0)  # the host model hands in the same fresh cells
                res_box[0] = mech.rosenbrock_host(
                    h_var, h_fix, h_temp, h_t[kk][0], h_t[kk][1], h_atol, h_rtol, wl.ipar,
                    wl.rpar, cfactor=h_cf, sun=h_sun, hstart=None if fresh else h_hs,
                    out=res_box[0])
                if not fresh:
                    h_hs.copy_(res_box[0].rstatus[1])  # the host model's warm start

            h2d = sum(nb(x) for x in (h_var, h_fix, h_temp, h_cf, h_sun, h_t[0][0], h_t[0][1],
                                      None if fresh else h_hs))
            d2h = nb(h_var) + 8 * n * 4 + 2 * n * 8 + n * 4
            api = ("kpp_b200_rosenbrock_host (pinned host arrays, chunked copies overlapped "
                   "with the integration, synchronous)")
        keep_var, keep_hs = h_var.clone(), h_hs.clone()
        e2e_step(args.warmup)  # warm the path, then replay the timed steps
        h_var.copy_(keep_var)
        h_hs.copy_(keep_hs)
        torch.cuda.synchronize()
        barrier()
        t_start = time.perf_counter()
        for k in range(args.warmup, total):
            e2e_step(k)
        ems = max_over_ranks((time.perf_counter() - t_start) * 1e3)
        barrier()
        same = bool(np.array_equal(h_var.numpy(), head.var_out))
        e2e = {"value": whole_job_rate(n, world, args.steps, ems), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": ems / args.steps, "api": api, "matches_device_run": same}

    sched_block = {"kind": "learned" if learned is not None else "plain"}
    if learned is not None:
        # the plan alone (features, network, binning) on the fresh batch
        var.copy_(var0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            sched.plan(var, temp, t_bounds[0][0], cfactor=cf, sun=sun, tend=t_bounds[0][1])
        e1.record(stream)
        torch.cuda.synchronize()
        sched_block.update({
            "speedup_vs_plain": learned.value / plain.value,
            "speedup_vs_plain_thread": (None if plain_thread is None
                                        else learned.value / plain_thread.value),
            "queue_cell_order": None if queued is None else {
                "what": "kpp_b200_rosenbrock_chain, Hstart = STEPMIN, cells in batch order "
                        f"({queue} queue): the work queue without the scheduler",
                "value": queued.value, "speedup_vs_plain": queued.value / plain.value,
                "bit_identical_to_plain": bool(np.array_equal(queued.var_out, plain.var_out)
                                               and np.array_equal(queued.ierr, plain.ierr)),
                "stats": queued.summary()},
            "speedup_vs_queue_cell_order": None if queued is None else learned.value / queued.value,
            "plan_ms": e0.elapsed_time(e1) / 3,
            "ierr_identical_to_plain": bool(np.array_equal(learned.ierr, plain.ierr)),
            "ceiling": None if ceiling is None else dict(
                ceiling_info, value=ceiling.value, speedup_vs_plain=ceiling.value / plain.value,
                learned_fraction_of_ceiling=learned.value / ceiling.value,
                stats=ceiling.summary()),
            "network": "78 features -> 3 x 256 GELU -> 2 (log10 Hstart, ln Nstp); BF16 "
                       "mma.sync GEMMs, FP32 accumulate; trained on the GPU by "
                       "kpp_b200.train_scheduler",
            "weights": (str(Path(sched.meta["source"]).resolve().relative_to(REPO))
                        if str(Path(sched.meta["source"]).resolve()).startswith(str(REPO))
                        else sched.meta["source"]),
            "training": TRAINING_SUMMARY.get(args.workload),
        })
    elif sched_note:
        sched_block["note"] = sched_note
    if fresh and args.accuracy_cells > 0:
        # cells spread over every cost level: evenly spaced positions of the
        # queue order by cost (the learned plan's order), else of the batch
        if learned is not None:
            sched.plan(var0, temp, t_bounds[0][0], cfactor=cf, sun=sun, tend=t_bounds[0][1],
                       hstart=torch.empty(n, dtype=torch.float64, device=dev),
                       order=(order_acc := torch.empty(n, dtype=torch.int32, device=dev)))
            pick = order_acc.cpu().numpy()
        else:
            pick = np.arange(n)
        cells = np.sort(pick[np.linspace(0, n - 1, min(args.accuracy_cells, n)).astype(np.int64)])
        ref, ref_ierr, tight_ms = tight_gpu(mech, wl, cells, dev)
        ok = ref_ierr == 1  # cells the tight solve finished
        A = lambda arm: accuracy(arm.var_out[:, cells[ok]], ref[:, ok], float(wl.atol[0]),
                                 float(wl.rtol[0])) if arm is not None and ok.any() else None
        acc = {"plain": A(plain), "learned": A(learned), "ceiling": A(ceiling),
               "oracle": f"FP64 Rodas4, RTOL {TIGHT_RTOL:g}, ATOL {TIGHT_ATOL:g}, at most 10^6 "
                         f"steps, on the GPU ({tight_ms / 1e3:.1f} s); cells evenly spaced "
                         f"over the cost order",
               "oracle_cells_ok": int(ok.sum()), "oracle_cells": int(ok.size),
               "oracle_ierr": sorted(set(int(x) for x in ref_ierr))}
        if pool is not None and args.accuracy_cpu_cells > 0:
            # the tight GPU solution against the CPU restatement of the
            # reference Rosenbrock on a subset of those cells
            sub = cells[np.linspace(0, len(cells) - 1, args.accuracy_cpu_cells).astype(np.int64)]
            cpu_ref, cpu_ierr = tight_reference(wl, sub, pool)
            idx = np.searchsorted(cells, sub)
            both = (cpu_ierr == 1) & ok[idx]
            if both.any():
                g, c = ref[:, idx[both]], cpu_ref[:, both]
                mask = np.abs(c) > 1e3 * TIGHT_ATOL
                acc["oracle_gpu_vs_cpu"] = {
                    "cells": int(both.sum()),
                    "max_rel_diff_above_1e3_atol": float((np.abs(g - c)[mask] / np.abs(c)[mask]).max())
                    if mask.any() else None}
        sched_block["accuracy_vs_fp64_rtol1e-10"] = acc

    nchunks = (n + (1 << 17) - 1) >> 17
    launches_learned = nchunks * (1 + 4) + 2 + 1
    result = {
        "metric": (METRIC if args.mech == "saprc99" else
                   f"{args.mech} cell-steps/s at {n} cells ({args.workload}, {method_title})"),
        "value": head.value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head.ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.mech} {args.workload} ({args.mode}) {method_title}, {n} "
                               f"cells per GPU, {wl.dt:.0f} s chemistry step, RTOL "
                               f"{wl.rtol[0]:g} ATOL {wl.atol[0]:g}",
                   "mode": args.mode, "cells_per_gpu": n, "chemistry_step_s": wl.dt,
                   "method": method_name, "scheduler": sched_block["kind"],
                   "queue": queue,
                   "parallelism": f"cell shards x{world}",
                   "kernel": {"thread": "thread per cell", "warp": "warp per cell"}[kernel],
                   "launch_shape": shape or {"kernel": kernel, "blocks_per_sm": 0,
                                             "source": "default (no tuning record)"},
                   "l2": "inputs larger than L2 (VAR alone %d MB)" % (wl.var.nbytes >> 20)},
        "impl": "kpp_b200",
        "gpu_launches": args.steps * (launches_learned if learned is not None
                                      else (2 if kernel == "warp" else 1)),
        "plain": dict(plain.summary(), kernel={"thread": "thread per cell",
                                                "warp": "warp per cell"}[plain_kernel]),
        "plain_thread": None if plain_thread is None else dict(
            plain_thread.summary(), kernel="thread per cell",
            bit_identical_to_plain=bool(np.array_equal(plain_thread.var_out, plain.var_out)
                                        and np.array_equal(plain_thread.ierr, plain.ierr))),
        "learned": learned.summary() if learned is not None else None,
        "scheduler": sched_block,
        "stats": head.summary(),
        "roofline": {"bound": "fp64", "achieved": achieved_tflops, "peak": peak_fma,
                     "unit": "TFLOP/s", "frac": achieved_tflops / peak_fma if peak_fma > 0 else None,
                     "traffic": traffic_per_launch,
                     "traffic_source": TRAFFIC_SOURCE[kernel],
                     "algorithmic_bytes_per_launch": ALGO_BYTES_PER_CELL_STEP * n,
                     "kernel_ms_per_launch": head.kernel_ms / args.steps,
                     "peak_source": "measured on this GPU by the DFMA throughput kernel "
                                    "(kpp_b200/csrc/kpp_util.cu); MEASURED_PEAKS.json has no FP64 figure",
                     "peak_mul_add_tflops": peak_muladd,
                     "flops_per_cell_step": flops / (n * args.steps)},
        "clocks": head.clocks,
        "e2e": e2e,
    }
    return result, wl


def run_diurnal(args, rank, world, local_rank):
    """The uneven-stiffness diurnal loop: every cell runs `--calls` chained
    600 s chemistry steps (the reference driver loop, TIME += DT, STEPMIN =
    Hexit) from its initial state.  Two forms, both replayed from CUDA graphs:
      per-step  one kpp_b200_rosenbrock launch per chemistry step (a device
                barrier between steps: every step waits for its slowest cell)
      persistent  one kpp_b200_rosenbrock_chain launch: each warp takes 32
                cells from the work queue and runs all their steps
      persistent_learned_order  the same launch, cells queued in the learned
                scheduler's cost order for the first (cold) step
    Results are compared bit for bit; `value` is the fastest form (named in
    `headline_form`)."""
    import torch
    from kpp_b200 import load, workloads
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    mech = load(args.mech)
    if args.queue != "tuned":
        mech.set_queue_lanes(args.queue == "lanes")
    # saprc99: the uneven-stiffness classes; another mechanism: its own
    # workload (small_strato: 72 x 1200 s steps of 4096 cells is config 1)
    wname = (args.workload if args.workload.endswith("classes") or args.mech != "saprc99"
             else "saprc99_classes")
    wl = workloads.for_mechanism(mech, wname, args.ncells, seed=shard_seed(rank))
    n, ncalls = wl.ncells, args.calls
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    var0 = D(wl.var)
    fix, temp = D(wl.fix), D(wl.temp)
    cf = D(wl.cfactor) if wl.cfactor is not None else None
    sun = D(wl.sun) if wl.sun is not None else None
    atol, rtol = D(wl.atol), D(wl.rtol)
    bounds = [tuple(D(x) for x in wl.driver_bounds(k)) for k in range(ncalls)]
    s = torch.cuda.Stream(dev)

    var_a = var0.clone()
    hs = torch.zeros(n, dtype=torch.float64, device=dev)
    ist_a = torch.zeros(8, n, dtype=torch.int32, device=dev)
    ierr_a = torch.ones(n, dtype=torch.int32, device=dev)
    box = [None]

    def per_step():
        var_a.copy_(var0)
        hs.zero_()  # first call: Hstart = RPAR[2] = 0, the default
        for k in range(ncalls):
            box[0] = o = mech.rosenbrock(var_a, fix, temp, bounds[k][0], bounds[k][1], atol,
                                         rtol, wl.ipar, wl.rpar, cfactor=cf, sun=sun, hstart=hs,
                                         out=box[0])
            hs.copy_(o.rstatus[1])
            if k == 0:
                ist_a.copy_(o.istatus)
                ierr_a.copy_(o.ierr)
            else:
                ist_a.add_(o.istatus)
                torch.where(ierr_a == 1, o.ierr, ierr_a, out=ierr_a)

    var_b = var0.clone()
    box_b = [None]

    def persistent():
        var_b.copy_(var0)
        box_b[0] = mech.rosenbrock_chain(var_b, fix, temp, bounds[0][0], wl.dt, ncalls, atol,
                                         rtol, wl.ipar, wl.rpar, cfactor=cf, sun=sun,
                                         out=box_b[0])

    # each form on each kernel the mechanism has (warp per cell where the
    # rate constants are fixed for a call); the kernel is chosen when the
    # form's graph is captured
    mech.set_kernel("warp")
    kernels = ["thread"] + (["warp"] if mech.kernel() == "warp" and sun is not None else [])
    forms = []
    for kn in kernels:
        forms.append((f"per_step_{kn}", per_step, kn))
        forms.append((f"persistent_{kn}", persistent, kn))
    wpath = Path(args.weights) if args.weights else (
        REPO / "kpp_b200" / "schedulers" / "saprc99_uniform95.npz")
    var_c = var0.clone()
    box_c = [None]
    if wpath.exists() and args.mech == "saprc99":
        from kpp_b200.scheduler import LearnedScheduler
        sched = LearnedScheduler.load(wpath, mech.nvar)
        order = torch.empty(n, dtype=torch.int32, device=dev)
        hs_plan = torch.empty(n, dtype=torch.float64, device=dev)

        def persistent_learned():
            # the scheduler's cost order for the loop's first (cold) step; its
            # Hstart is not used, so the results stay those of the other forms
            var_c.copy_(var0)
            sched.plan(var_c, temp, bounds[0][0], cfactor=cf, sun=sun, tend=bounds[0][1],
                       hstart=hs_plan, order=order)
            box_c[0] = mech.rosenbrock_chain(var_c, fix, temp, bounds[0][0], wl.dt, ncalls,
                                             atol, rtol, wl.ipar, wl.rpar, cfactor=cf, sun=sun,
                                             order=order, out=box_c[0])

        forms.append(("persistent_learned_order", persistent_learned, kernels[-1]))

    # inputs smaller than L2 (126 MB): a 256 MB buffer written between the
    # timed loops
    small = wl.var.nbytes < (192 << 20)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if small else None
    results = {}
    outs = {}
    for name, body, kn in forms:
        mech.set_kernel(kn)
        with torch.cuda.stream(s):
            body()  # allocates the library workspace of stream s before capture
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            body()
        # replay() launches on the current stream: time on that same stream
        with torch.cuda.stream(s):
            for _ in range(args.warmup):
                g.replay()
            torch.cuda.synchronize()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
            with ClockSampler(local_rank) as clk:
                for e0, e1 in evs:
                    if flush is not None:
                        flush.fill_(1)  # L2 flushed between timed loops, outside the events
                    e0.record(s)
                    g.replay()
                    e1.record(s)
                torch.cuda.synchronize()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
        if world > 1:
            ms = reduce_max(ms, dev)
        results[name] = {"kernel": {"thread": "thread per cell", "warp": "warp per cell"}[kn],
                         "ms_per_loop": ms / args.steps,
                         "value": whole_job_rate(n * ncalls, world, args.steps, ms),
                         "clocks": clk.summary()}
        # the state after the form's last replay, for the bit-for-bit check
        if name.startswith("per_step"):
            outs[name] = (var_a.clone(), ist_a.clone(), ierr_a.clone(), box[0].rstatus.clone())
        else:
            o = box_c[0] if name == "persistent_learned_order" else box_b[0]
            v = var_c if name == "persistent_learned_order" else var_b
            outs[name] = (v.clone(), o.istatus.clone(), o.ierr.clone(), o.rstatus.clone())
        del g
    mech.set_kernel("auto")
    ob = box_b[0]
    ref_out = next(iter(outs.values()))
    same = all(all(torch.equal(a, b) for a, b in zip(ref_out, o)) for o in outs.values())
    nstp = ob.istatus[2].to(torch.float64)
    sza = wl.meta.get("sza")
    classes = {}
    if sza is not None:
        for nm, lo, hi in (("day", 0, 85), ("terminator", 85, 95), ("night", 95, 181)):
            mask = D(((sza >= lo) & (sza < hi)).astype(np.bool_))
            if bool(mask.any()):
                classes[nm] = float(nstp[mask].mean() / ncalls)
    head = max(results.values(), key=lambda r: r["value"])
    head_name = [k for k, v in results.items() if v is head][0]
    # the comparison: the faster of the one-launch-per-step forms
    best_step = max((k for k in results if k.startswith("per_step")),
                    key=lambda k: results[k]["value"])
    # the loop's final state against the tight solution of the whole loop
    # (at most 1024 cells: each runs ncalls tight chemistry steps)
    acc = (accuracy_block(mech, wl, var_b.cpu().numpy(), n, ncalls, dev,
                          min(args.accuracy_cells, 1024)) if args.accuracy_cells > 0 else None)
    return {
        "metric": f"{args.mech} cell-steps/s, {n} cells"
                  + (" of uneven stiffness" if sza is not None else "")
                  + f", {ncalls}-step diurnal loop (persistent work queue vs one launch per step)",
        "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_loop"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.mech} {wname}: "
                               + ("40 % day, 40 % night, 20 % within 5 deg of the terminator; "
                                  if sza is not None else "start times over a whole day, SUN "
                                  "from Update_SUN(TIME); ")
                               + f"{ncalls} x {wl.dt:.0f} s Rodas3 steps, RTOL {wl.rtol[0]:g} "
                                 f"ATOL {wl.atol[0]:g}; one step = one diurnal loop of every cell",
                   "cells_per_gpu": n, "graph": "both forms replayed from CUDA graphs",
                   "queue": "lanes" if mech.queue_lanes() else "warps",
                   "l2": ("inputs smaller than L2: 256 MB written between timed loops, "
                          "outside the timed events" if small else "inputs larger than L2")},
        "impl": "kpp_b200", "gpu_launches": args.steps,
        "forms": results, "headline_form": head_name,
        "per_step_baseline": best_step,
        "speedup_vs_per_step": {k: v["value"] / results[best_step]["value"]
                                for k, v in results.items()},
        "bit_identical": bool(same),
        "internal_steps_per_cell_step": float(nstp.mean() / ncalls),
        "internal_steps_per_cell_step_by_class": classes,
        "ierr_ok_fraction": float((ob.ierr == 1).to(torch.float64).mean()),
        "accuracy_vs_fp64_rtol1e-10": acc,
        "clocks": head["clocks"],
    }


def run_adjoint(args, rank, world, local_rank):
    """The Rosenbrock discrete adjoint (int/rosenbrock_adj.c) on the
    fresh-cell workload, in the library built on KPP's own generator: every
    timed step integrates the same fresh batch forward over one chemistry
    step and back with kpp_b200_rosenbrock_adj (one launch), NADJ adjoint
    vectors per cell."""
    import torch
    from kpp_b200 import Mechanism, workloads
    from kpp_b200 import build as kbuild
    from kpp_b200.build import LIB

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    path = kbuild.library_path(args.mech, "kpp")
    if not path.exists():
        raise SystemExit(f"{path} not built: the adjoint is in the generator-route library")
    mech = Mechanism(args.mech, path=path)
    wl = workloads.for_mechanism(mech, args.workload, args.adj_cells, seed=shard_seed(rank))
    n = wl.ncells
    kind, ic, rc, nadj, bufsize = mode_integrator(args)
    name = integrator_name(kind, ic[2])
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    lam_h = np.random.default_rng(7).standard_normal((nadj * mech.nvar, n))
    var0, lam0 = D(wl.var), D(lam_h)
    var, lam = var0.clone(), lam0.clone()
    fix, temp = D(wl.fix), D(wl.temp)
    cf = D(wl.cfactor) if wl.cfactor is not None else None
    sun = D(wl.sun) if wl.sun is not None else None
    atol, rtol = D(wl.atol), D(wl.rtol)
    t0, t1 = (D(x) for x in wl.step_bounds(0))
    stream = torch.cuda.current_stream(dev)
    work = torch.empty(int(mech.lib.kpp_b200_rosenbrock_adj_work_bytes(n, nadj, bufsize, ic[7]))
                       // 8, dtype=torch.float64, device=dev)
    box = [None]
    small = wl.var.nbytes + lam_h.nbytes < (192 << 20)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev) if small else None

    def step():
        var.copy_(var0)
        lam.copy_(lam0)
        box[0] = mech.rosenbrock_adj(var, fix, temp, t0, t1, atol, rtol, lam, ic, rc,
                                     bufsize=bufsize, cfactor=cf, sun=sun, out=box[0], work=work)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    stats = []
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for e0, e1 in evs:
            var.copy_(var0)
            lam.copy_(lam0)
            if flush is not None:
                flush.fill_(1)
            e0.record(stream)
            box[0] = mech.rosenbrock_adj(var, fix, temp, t0, t1, atol, rtol, lam, ic, rc,
                                         bufsize=bufsize, cfactor=cf, sun=sun, out=box[0],
                                         work=work)
            e1.record(stream)
            stats.append(box[0].istatus.sum(dim=1))
        torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    if world > 1:
        ms = reduce_max(ms, dev)
    ist = torch.stack(stats).sum(dim=0).cpu().numpy().astype(np.int64)
    nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng = ist.tolist()
    ierr = box[0].ierr.cpu().numpy()
    # FP64 work from the counters, a lower bound: Fun, Jacobian, LU and
    # (transposed) solves of both passes; the Hessian and its products are
    # not counted
    opsd = {}
    hdr = REPO / "kpp_b200" / "_gen" / f"{args.mech}.cuh"
    for line in hdr.read_text().splitlines() if hdr.exists() else []:
        if line.startswith("#define KPP_OPS_"):
            _, kk, v = line.split()
            opsd[kk[8:].lower()] = int(v)
    flops = (nfun * opsd.get("fun", 0) + njac * opsd.get("jac", 0)
             + ndec * opsd.get("decomp", 0) + nsol * opsd.get("solve", 0))
    achieved = flops / (ms / 1e3) / 1e12
    peak_fma, _ = fp64_peak(LIB / "libkpp_b200_util.so")

    e2e = None
    if args.e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        h = {k: pin(v) for k, v in (("var", wl.var), ("lam", lam_h), ("fix", wl.fix),
                                    ("temp", wl.temp), ("t0", wl.step_bounds(0)[0]),
                                    ("t1", wl.step_bounds(0)[1]), ("atol", wl.atol),
                                    ("rtol", wl.rtol))}
        if wl.cfactor is not None:
            h["cf"] = pin(wl.cfactor)
        if wl.sun is not None:
            h["sun"] = pin(wl.sun)
        h_out = {"var": torch.empty_like(h["var"]).pin_memory(),
                 "lam": torch.empty_like(h["lam"]).pin_memory(),
                 "ist": torch.empty(8, n, dtype=torch.int32).pin_memory(),
                 "rst": torch.empty(3, n, dtype=torch.float64).pin_memory(),
                 "ierr": torch.empty(n, dtype=torch.int32).pin_memory()}
        d = {k: torch.empty_like(v, device=dev) for k, v in h.items()}
        ebox = [None]

        def e2e_step():
            for k, v in h.items():
                d[k].copy_(v, non_blocking=True)
            ebox[0] = o = mech.rosenbrock_adj(d["var"], d["fix"], d["temp"], d["t0"], d["t1"],
                                              d["atol"], d["rtol"], d["lam"], ic, rc,
                                              bufsize=bufsize, cfactor=d.get("cf"),
                                              sun=d.get("sun"), out=ebox[0], work=work)
            h_out["var"].copy_(d["var"], non_blocking=True)
            h_out["lam"].copy_(d["lam"], non_blocking=True)
            h_out["ist"].copy_(o.istatus, non_blocking=True)
            h_out["rst"].copy_(o.rstatus, non_blocking=True)
            h_out["ierr"].copy_(o.ierr, non_blocking=True)
            stream.synchronize()

        e2e_step()
        torch.cuda.synchronize()
        t_start = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        ems = (time.perf_counter() - t_start) * 1e3
        if world > 1:
            ems = reduce_max(ems, dev)
        nb = lambda x: x.numel() * x.element_size()
        e2e = {"value": whole_job_rate(n, world, args.steps, ems), "unit": UNIT,
               "h2d_bytes_per_step": int(sum(nb(v) for v in h.values())),
               "d2h_bytes_per_step": int(sum(nb(v) for v in h_out.values())),
               "ms_per_step": ems / args.steps,
               "api": "Mechanism.rosenbrock_adj (kpp_b200_rosenbrock_adj), pinned host arrays "
                      "copied in and out every step",
               "matches_device_run": bool(np.array_equal(h_out["lam"].numpy(),
                                                         lam.cpu().numpy()))}

    return {
        "metric": f"{args.mech} cell-steps/s at {n} cells, Rosenbrock discrete adjoint "
                  f"{name}, NADJ {nadj} (int/rosenbrock_adj.c)",
        "value": whole_job_rate(n, world, args.steps, ms), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"{args.mech} {args.workload} (fresh) {name} forward and "
                               f"discrete adjoint, {n} cells per GPU, {wl.dt:.0f} s chemistry "
                               f"step, RTOL {wl.rtol[0]:g} ATOL {wl.atol[0]:g}, NADJ {nadj}, "
                               f"{bufsize} trajectory entries per cell",
                   "mode": "adj", "cells_per_gpu": n, "method": name, "nadj": nadj,
                   "bufsize": bufsize, "library": path.name,
                   "work_bytes": int(work.numel() * 8),
                   "parallelism": f"cell shards x{world}",
                   "l2": ("inputs smaller than L2: 256 MB written between timed steps, outside "
                          "the timed events" if small else "inputs larger than L2")},
        "impl": "kpp_b200", "gpu_launches": args.steps,
        "stats": {"internal_steps_per_cell_step": nstp / (n * args.steps),
                  "ierr_ok_fraction": float((ierr == 1).mean()),
                  "istatus_sum": dict(zip(["nfun", "njac", "nstp", "nacc", "nrej", "ndec",
                                           "nsol", "nsng"], map(int, ist)))},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak_fma, "unit": "TFLOP/s",
                     "frac": achieved / peak_fma if peak_fma > 0 else None, "traffic": None,
                     "achieved_note": "lower bound: Fun, Jacobian, LU and solves of both "
                                      "passes; Hessian evaluations and products not counted",
                     "peak_source": "measured on this GPU by the DFMA throughput kernel "
                                    "(kpp_b200/csrc/kpp_util.cu)"},
        "clocks": clk.summary(),
        "e2e": e2e,
    }, wl


SDIRK_NAMES = {1: "Sdirk2a", 2: "Sdirk2b", 3: "Sdirk3a", 4: "Sdirk4a", 5: "Sdirk4b"}
RK_NAMES = {0: "Radau-2A", 1: "Radau-2A", 2: "Lobatto-3C", 3: "Gauss", 4: "Radau-1A",
            5: "Lobatto-3A"}
# kind: (entry of kpp_b200.Mechanism, reference file, method names, default name)
ADJ_NAMES = {0: "Rodas3", 1: "Ros2", 2: "Ros3", 3: "Ros4", 4: "Rodas3", 5: "Rodas4",
             7: "Rodas3_1"}
INTEGRATORS = {"sdirk": ("sdirk", "int/sdirk.c", SDIRK_NAMES, "Sdirk2a"),
               "rk": ("runge_kutta", "int/runge_kutta.c", RK_NAMES, "Radau-2A"),
               "adj": ("rosenbrock_adj", "int/rosenbrock_adj.c", ADJ_NAMES, "Rodas3")}


def integrator_controls(kind: str, method: int):
    """(kind, ICNTRL, RCNTRL) for the workload's scalar tolerances and the
    given method, every other control at its default; for Runge-Kutta with
    INTEGRATE's SDIRK error estimator (int/runge_kutta.c:131-139)."""
    ic, rc = [0] * 20, [0.0] * 20
    ic[1], ic[2] = 1, method
    if kind == "rk":
        ic[9] = 1
    return kind, ic, rc


def mode_integrator(args):
    """(kind, ICNTRL, RCNTRL) of the --mode sdirk / rk runs, else None."""
    if args.mode == "sdirk":
        return integrator_controls("sdirk", args.sdirk_method)
    if args.mode == "rk":
        return integrator_controls("rk", args.rk_method)
    if args.mode == "adj":
        # (kind, ICNTRL, RCNTRL, NADJ, bufsize): the discrete adjoint of the
        # method, ICNTRL[3] = 0 (the step limit is bufsize - 1)
        kind, ic, rc = integrator_controls("adj", args.adj_method)
        return kind, ic, rc, args.nadj, args.adj_bufsize
    return None


def integrator_name(kind: str, method: int) -> str:
    names, default = INTEGRATORS[kind][2], INTEGRATORS[kind][3]
    return names.get(method, default)


def run_integrator(args, rank, world, local_rank, kind: str):
    """The SDIRK (int/sdirk.c) or Runge-Kutta (int/runge_kutta.c)
    integrator on the fresh-cell workload: every timed step integrates the
    same fresh batch over one chemistry step with kpp_b200_sdirk /
    kpp_b200_runge_kutta (one launch)."""
    import torch
    from kpp_b200 import load, workloads
    from kpp_b200.build import LIB

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    mech = load(args.mech)
    wl = workloads.for_mechanism(mech, args.workload, args.ncells, seed=shard_seed(rank))
    n = wl.ncells
    method = args.sdirk_method if kind == "sdirk" else args.rk_method
    _, ic, rc = integrator_controls(kind, method)
    name = integrator_name(kind, method)
    entry_name, source = INTEGRATORS[kind][0], INTEGRATORS[kind][1]
    entry = getattr(mech, entry_name)
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    var0 = D(wl.var)
    var = var0.clone()
    fix, temp = D(wl.fix), D(wl.temp)
    cf = D(wl.cfactor) if wl.cfactor is not None else None
    sun = D(wl.sun) if wl.sun is not None else None
    atol, rtol = D(wl.atol), D(wl.rtol)
    t0, t1 = (D(x) for x in wl.step_bounds(0))
    stream = torch.cuda.current_stream(dev)
    box = [None]

    def step():
        var.copy_(var0)  # the same fresh batch every step
        box[0] = entry(var, fix, temp, t0, t1, atol, rtol, ic, rc, cfactor=cf, sun=sun,
                            out=box[0])

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for k in range(args.steps):
            var.copy_(var0)
            kev[k][0].record(stream)
            box[0] = entry(var, fix, temp, t0, t1, atol, rtol, ic, rc, cfactor=cf, sun=sun,
                                out=box[0])
            kev[k][1].record(stream)
            stats.append(box[0].istatus.sum(dim=1))
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        ms = reduce_max(ms, dev)
    kernel_ms = sum(a.elapsed_time(b) for a, b in kev)
    ist = torch.stack(stats).sum(dim=0).cpu().numpy().astype(np.int64)
    nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng = ist.tolist()
    ierr = box[0].ierr.cpu().numpy()
    var_dev = var.cpu().numpy()
    acc = (accuracy_block(mech, wl, var_dev, n, 1, dev, args.accuracy_cells)
           if args.accuracy_cells > 0 else None)

    # FP64 work from the counters.  SDIRK: Fun per Newton iteration, Jac +
    # LU per factorisation, a solve per Newton iteration and error estimate.
    # Runge-Kutta (a lower bound: the SDIRK estimator's solves and the
    # estimator's extra Fun calls that ISTATUS does not count are left out):
    # the counted Fun calls plus three stage evaluations per Newton iteration
    # (one RK_Solve each), a real and a complex LU per factorisation, a real
    # and a complex solve per Newton iteration.
    opsd = {}
    for hname in (f"{args.mech}.cuh", f"{args.mech}_cmplx.cuh"):
        hdr = REPO / "kpp_b200" / "_gen" / hname
        for line in hdr.read_text().splitlines() if hdr.exists() else []:
            if line.startswith("#define KPP_OPS_"):
                _, kk, v = line.split()
                opsd[kk[8:].lower()] = int(v)
    if kind == "sdirk":
        flops = (nfun * opsd.get("fun", 0) + njac * opsd.get("jac", 0)
                 + ndec * opsd.get("decomp", 0) + nsol * opsd.get("solve", 0))
    else:
        flops = ((nfun + 3 * nsol) * opsd.get("fun", 0) + njac * opsd.get("jac", 0)
                 + ndec * (opsd.get("decomp", 0) + opsd.get("decomp_cmplx", 0))
                 + nsol * (opsd.get("solve", 0) + opsd.get("solve_cmplx", 0)))
    achieved = flops / (kernel_ms / 1e3) / 1e12
    peak_fma, _ = fp64_peak(LIB / "libkpp_b200_util.so")

    e2e = None
    if args.e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        h = {k: pin(v) for k, v in (("var", wl.var), ("fix", wl.fix), ("temp", wl.temp),
                                    ("t0", wl.step_bounds(0)[0]), ("t1", wl.step_bounds(0)[1]),
                                    ("atol", wl.atol), ("rtol", wl.rtol))}
        if wl.cfactor is not None:
            h["cf"] = pin(wl.cfactor)
        if wl.sun is not None:
            h["sun"] = pin(wl.sun)
        h_out = {"var": torch.empty_like(h["var"]).pin_memory(),
                 "ist": torch.empty(8, n, dtype=torch.int32).pin_memory(),
                 "rst": torch.empty(3, n, dtype=torch.float64).pin_memory(),
                 "ierr": torch.empty(n, dtype=torch.int32).pin_memory()}
        d = {k: torch.empty_like(v, device=dev) for k, v in h.items()}
        ebox = [None]

        def e2e_step():
            for k, v in h.items():
                d[k].copy_(v, non_blocking=True)
            ebox[0] = o = entry(d["var"], d["fix"], d["temp"], d["t0"], d["t1"], d["atol"],
                                     d["rtol"], ic, rc, cfactor=d.get("cf"), sun=d.get("sun"),
                                     out=ebox[0])
            h_out["var"].copy_(d["var"], non_blocking=True)
            h_out["ist"].copy_(o.istatus, non_blocking=True)
            h_out["rst"].copy_(o.rstatus, non_blocking=True)
            h_out["ierr"].copy_(o.ierr, non_blocking=True)
            stream.synchronize()

        e2e_step()
        torch.cuda.synchronize()
        t_start = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        ems = (time.perf_counter() - t_start) * 1e3
        if world > 1:
            ems = reduce_max(ems, dev)
        nb = lambda x: x.numel() * x.element_size()
        e2e = {"value": whole_job_rate(n, world, args.steps, ems), "unit": UNIT,
               "h2d_bytes_per_step": int(sum(nb(v) for v in h.values())),
               "d2h_bytes_per_step": int(sum(nb(v) for v in h_out.values())),
               "ms_per_step": ems / args.steps,
               "api": f"Mechanism.{entry_name} (kpp_b200_{entry_name}), pinned host arrays "
                      "copied in and out every step",
               "matches_device_run": bool(np.array_equal(h_out["var"].numpy(), var_dev))}

    return {
        "metric": f"{args.mech} cell-steps/s at {n} cells, {kind.upper()} {name} ({source})",
        "value": whole_job_rate(n, world, args.steps, ms), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"{args.mech} {args.workload} (fresh) {name}, {n} cells per GPU, "
                               f"{wl.dt:.0f} s chemistry step, RTOL {wl.rtol[0]:g} ATOL "
                               f"{wl.atol[0]:g}, other controls at {source} defaults",
                   "mode": kind, "cells_per_gpu": n, "method": name,
                   "parallelism": f"cell shards x{world}",
                   "l2": "inputs larger than L2 (VAR alone %d MB)" % (wl.var.nbytes >> 20)},
        "impl": "kpp_b200", "gpu_launches": args.steps,
        "stats": {"internal_steps_per_cell_step": nstp / (n * args.steps),
                  "rejected_step_rate": nrej / max(nstp, 1),
                  "ierr_ok_fraction": float((ierr == 1).mean()),
                  "istatus_sum": dict(zip(["nfun", "njac", "nstp", "nacc", "nrej", "ndec",
                                           "nsol", "nsng"], map(int, ist)))},
        "accuracy_vs_fp64_rtol1e-10": acc,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak_fma, "unit": "TFLOP/s",
                     "frac": achieved / peak_fma if peak_fma > 0 else None, "traffic": None,
                     "kernel_ms_per_launch": kernel_ms / args.steps,
                     "flops_per_cell_step": flops / (n * args.steps),
                     "peak_source": "measured on this GPU by the DFMA throughput kernel "
                                    "(kpp_b200/csrc/kpp_util.cu)"},
        "clocks": clk.summary(),
        "e2e": e2e,
    }, wl


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--mode", choices=["fresh", "chain", "diurnal", "sdirk", "rk", "adj"],
                    default="fresh")
    ap.add_argument("--sdirk-method", type=int, default=0,
                    help="ICNTRL[2] of the SDIRK mode (0: INTEGRATE's default, Sdirk2a)")
    ap.add_argument("--rk-method", type=int, default=0,
                    help="ICNTRL[2] of the Runge-Kutta mode (0: INTEGRATE's default, Radau-2A)")
    ap.add_argument("--calls", type=int, default=24, help="chemistry steps of a diurnal loop")
    ap.add_argument("--adj-method", type=int, default=0,
                    help="--mode adj: ICNTRL[2] of int/rosenbrock_adj.c (0 Rodas3)")
    ap.add_argument("--nadj", type=int, default=1, help="--mode adj: adjoint vectors per cell")
    ap.add_argument("--adj-bufsize", type=int, default=200,
                    help="--mode adj: trajectory entries per cell (step limit bufsize - 1)")
    ap.add_argument("--adj-cells", type=int, default=32768, help="--mode adj: cells per GPU")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["kpp_b200", "reference"], default="kpp_b200")
    ap.add_argument("--mech", default="saprc99")
    ap.add_argument("--workload", default="saprc99_uniform95")
    ap.add_argument("--ncells", type=int, default=1 << 20)
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--kernel", choices=["auto", "thread", "warp"], default="auto")
    ap.add_argument("--queue", choices=["tuned", "lanes", "warps"], default="tuned",
                    help="work-queue granularity of the queue, learned and ceiling arms: each "
                         "warp takes 32 cells at a time, or each lane one (its cells advancing "
                         "step by step together); default: the autotuner's record, else the "
                         "library's default (lanes)")
    ap.add_argument("--scheduler", choices=["learned", "plain"], default="learned")
    ap.add_argument("--weights", default=None, help="trained scheduler (.npz)")
    ap.add_argument("--accuracy-cells", type=int, default=4096,
                    help="cells compared with the FP64 RTOL 1e-10 solution (on the GPU)")
    ap.add_argument("--accuracy-cpu-cells", type=int, default=64,
                    help="of those, cells also solved by the CPU oracle as a cross-check")
    ap.add_argument("--no-plain-thread", dest="plain_thread", action="store_false",
                    help="skip the thread-per-cell plain arm beside the automatic plain arm")
    ap.add_argument("--no-queue-arm", dest="queue_arm", action="store_false",
                    help="skip the work-queue arm in cell order with the plain controls")
    ap.add_argument("--no-ceiling", dest="ceiling", action="store_false",
                    help="skip the ceiling arm (best starting step, true cost order)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    procs = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return 0
        ctx = mp.get_context("spawn")
        from kpp_b200 import workloads
        sys.path.insert(0, str(REPO / "tests"))
        from oracle_lib import OracleLib
        # the workload from the reference's own generated model (species,
        # #INITVALUES, CFACTOR): this arm maps no library of kpp_b200
        wl = workloads.for_mechanism(OracleLib(args.mech), args.workload,
                                     args.adj_cells if args.mode == "adj" else args.ncells,
                                     seed=workloads.SEED_EVAL)
        integ = mode_integrator(args)
        with ctx.Pool(procs) as pool:
            n_sample, _ = calibrated_sample(wl, procs, pool, target_s=min(args.cpu_seconds, 20.0),
                                            integ=integ)
            for _ in range(args.warmup and 1):
                cpu_reference_rate(wl, max(procs * 4, 64), procs, "", pool, integ)
            rates, walls = [], []
            for _ in range(args.steps):
                r, w = cpu_reference_rate(wl, n_sample, procs, "", pool, integ)
                rates.append(r)
                walls.append(w)
            # the same code built -O3 -march=x86-64-v3 (FMA contraction)
            rate_o3, _ = cpu_reference_rate(wl, n_sample, procs, "_O3", pool, integ)
        v = statistics.median(rates)
        metric = METRIC
        source = "int/rosenbrock.c"
        if integ:
            kind = integ[0]
            source = INTEGRATORS[kind][1]
            name = integrator_name(kind, integ[1][2])
            metric = (f"{args.mech} cell-steps/s at {args.ncells} cells, {kind.upper()} {name} "
                      f"({source})")
            if kind == "adj":
                metric = (f"{args.mech} cell-steps/s at {args.adj_cells} cells, Rosenbrock "
                          f"discrete adjoint {name}, NADJ {args.nadj} ({source})")
        line = {"metric": metric, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(walls),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": {"workload": f"{args.mech} {args.workload} plain, reference controls, chemistry "
                                       f"steps, RTOL 1e-3 ATOL 1e-2; each step a sample of "
                                       f"{n_sample} of the {wl.ncells} cells"},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": "reference",
                                 "sample": f"{n_sample} cells x 1 chemistry step per timed step, "
                                           f"{procs} processes, KPP-generated C + {source} "
                                           f"(gcc -O), host CPU {host_cpu_model()}",
                                 "value_O3": rate_o3,
                                 "value_O3_build": "the same sources, gcc -O3 -march=x86-64-v3 "
                                                   "-ffp-contract=fast (built where the reference "
                                                   "sources are, run on this host: x86-64-v3 rather "
                                                   "than -march=native)"},
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
    integ = mode_integrator(args)
    if args.mode == "diurnal":
        if pool is not None:
            pool.close()
            pool = None
        result = run_diurnal(args, rank, world, local_rank)
    elif args.mode == "adj":
        result, wl = run_adjoint(args, rank, world, local_rank)
    elif integ is not None:
        result, wl = run_integrator(args, rank, world, local_rank, integ[0])
    else:
        result, wl = run_cuda_arm(args, rank, world, local_rank, pool)
    if pool is not None:
        n_sample, _ = calibrated_sample(wl, procs, pool, target_s=args.cpu_seconds, integ=integ)
        rate, wall = cpu_reference_rate(wl, n_sample, procs, "", pool, integ)
        rate_o3, wall_o3 = cpu_reference_rate(wl, n_sample, procs, "_O3", pool, integ)
        pool.close()
        source = INTEGRATORS[integ[0]][1] if integ else "int/rosenbrock.c"
        result["cpu_baseline"] = {
            "value": rate, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{n_sample} cells x 1 chemistry step of the same workload, {procs} processes "
                      f"(reference KPP-generated C + {source}, gcc -O), {wall:.1f} s wall, "
                      f"host CPU {host_cpu_model()}",
            "value_O3": rate_o3,
            "value_O3_build": f"the same sources, gcc -O3 -march=x86-64-v3 -ffp-contract=fast "
                              f"({wall_o3:.1f} s wall; x86-64-v3 rather than -march=native: "
                              f"built on another host than it runs on)"}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
