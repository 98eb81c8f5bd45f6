"""Learned cell scheduler: Python side of libkpp_b200_sched.so (include/kpp_sched.h).

A small MLP reads a cell's state (log10 concentrations, T, ln CFACTOR, SUN,
ln dt) and predicts, for one chemistry step, a starting step Hstart and the
step count the integrator will need.  kpp_sched_plan turns the predictions
into per-cell Hstart (RPAR[2] of each cell's call) and a work-queue order with
the most expensive cells first, so the 32 cells of a warp cost about the
same; kpp_b200_rosenbrock_chain then integrates the cells in that order.  The
Rosenbrock controller is untouched: it still accepts or rejects every step.

Training data are logged from the plain GPU integrator: every training cell
is integrated once per candidate Hstart, and the tuple is (features, log10 of
the candidate that needed the fewest steps, ln of that step count).  The
network is trained by the library's own kernels (BF16 tensor-core GEMMs with
FP32 accumulation, backward pass, Adam).  No part of the reference is learned;
KPP starts every call at Hstart = STEPMIN (int/rosenbrock.c:102-104).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np
import torch

from .build import LIB

_vp = ctypes.c_void_p
_f = ctypes.c_float
_d = ctypes.c_double
_i = ctypes.c_int
_l = ctypes.c_long

WIDTH, NHIDDEN, NOUT = 256, 3, 2
# candidate Hstart values of the tuple logging: half decades 1e-6 .. 1e-2 s
CANDIDATES = tuple(float(10.0 ** e) for e in np.arange(-6.0, -1.99, 0.5))
FLOOR = 1e-20


class SchedError(RuntimeError):
    pass


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = LIB / "libkpp_b200_sched.so"
        if not path.exists():
            raise SchedError(f"{path} is missing: run python -m kpp_b200.build")
        L = ctypes.CDLL(str(path))
        L.kpp_sched_last_error.restype = ctypes.c_char_p
        L.kpp_sched_mlp_create.restype = _vp
        L.kpp_sched_mlp_create.argtypes = [_i] * 5
        L.kpp_sched_mlp_destroy.argtypes = [_vp]
        L.kpp_sched_mlp_param_count.restype = _l
        L.kpp_sched_mlp_param_count.argtypes = [_vp]
        for fn in ("kpp_sched_mlp_set_params", "kpp_sched_mlp_get_params",
                   "kpp_sched_mlp_get_params_bf16", "kpp_sched_mlp_get_grads"):
            getattr(L, fn).argtypes = [_vp, _vp]
        L.kpp_sched_mlp_set_scaling.argtypes = [_vp] * 5
        L.kpp_sched_mlp_forward.argtypes = [_vp, _i, _vp, _l, _vp, _vp]
        L.kpp_sched_mlp_loss_grad.argtypes = [_vp, _i, _vp, _l, _vp, _vp, _vp]
        L.kpp_sched_mlp_adam.argtypes = [_vp, _f, _f, _f, _f, _vp]
        L.kpp_sched_gather_columns.argtypes = [_i, _i, _vp, _vp, _l, _vp, _l, _vp]
        L.kpp_sched_features.argtypes = [_vp, _i, _i, _i] + [_vp] * 6 + [_d, _vp, _l, _vp]
        L.kpp_sched_plan.argtypes = ([_vp, _i, _i, _i] + [_vp] * 6
                                     + [_d, _d, _d, _i, _f, _f, _vp, _vp, _vp, _vp])
        _lib = L
    return _lib


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else _vp(t.data_ptr())


def _stream(dev):
    return _vp(torch.cuda.current_stream(dev).cuda_stream)


def _check(rc: int):
    if rc != 0:
        raise SchedError(lib().kpp_sched_last_error().decode())


def host_features(var: np.ndarray, temp, cfactor, sun, dt) -> np.ndarray:
    """The feature definition of kpp_sched_features, in float64 on the host
    ([nin][ncells]); used for the standardisation statistics."""
    n = var.shape[1]
    f = np.empty((var.shape[0] + 4, n))
    f[:-4] = np.log10(np.maximum(var, FLOOR))
    f[-4] = temp
    f[-3] = np.log(cfactor) if cfactor is not None else 0.0
    f[-2] = sun if sun is not None else 0.0
    f[-1] = math.log(dt)
    return f


class Mlp:
    """The network and its training buffers on the current CUDA device."""

    def __init__(self, nin: int, width: int = WIDTH, nhidden: int = NHIDDEN, nout: int = NOUT,
                 max_batch: int = 8192):
        if not torch.cuda.is_available():
            raise SchedError("the learned scheduler runs on the GPU only (no CPU fallback)")
        self.nin, self.width, self.nhidden, self.nout = nin, width, nhidden, nout
        self.max_batch = max_batch
        self.h = lib().kpp_sched_mlp_create(nin, width, nhidden, nout, max_batch)
        if not self.h:
            raise SchedError(lib().kpp_sched_last_error().decode())
        self.nparam = lib().kpp_sched_mlp_param_count(self.h)
        self.dev = torch.device("cuda", torch.cuda.current_device())
        self._loss = torch.zeros(1, dtype=torch.float32, device=self.dev)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().kpp_sched_mlp_destroy(h)
            self.h = None

    def shapes(self):
        fin = [self.nin] + [self.width] * self.nhidden
        fout = [self.width] * self.nhidden + [self.nout]
        return list(zip(fout, fin))

    def _host_vec(self, fn) -> np.ndarray:
        a = np.empty(self.nparam, dtype=np.float32)
        _check(fn(self.h, _vp(a.ctypes.data)))
        return a

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.nparam:
            raise SchedError(f"expected {self.nparam} parameters, got {p.size}")
        _check(lib().kpp_sched_mlp_set_params(self.h, _vp(p.ctypes.data)))

    def params(self) -> np.ndarray:
        return self._host_vec(lib().kpp_sched_mlp_get_params)

    def params_bf16(self) -> np.ndarray:
        return self._host_vec(lib().kpp_sched_mlp_get_params_bf16)

    def grads(self) -> np.ndarray:
        return self._host_vec(lib().kpp_sched_mlp_get_grads)

    def set_scaling(self, in_mu, in_sd, out_mu, out_sd):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (in_mu, in_sd, out_mu, out_sd)]
        _check(lib().kpp_sched_mlp_set_scaling(self.h, *[_vp(a.ctypes.data) for a in arrs]))

    def forward(self, x: torch.Tensor, n: Optional[int] = None) -> torch.Tensor:
        """x: BF16 [nin][ld] (feature-major).  Returns [n][nout] FP32."""
        n = x.shape[1] if n is None else n
        out = torch.empty(n, self.nout, dtype=torch.float32, device=x.device)
        _check(lib().kpp_sched_mlp_forward(self.h, n, _ptr(x), x.shape[1], _ptr(out),
                                           _stream(x.device)))
        return out

    def loss_grad(self, x: torch.Tensor, y: torch.Tensor, n: Optional[int] = None) -> torch.Tensor:
        n = x.shape[1] if n is None else n
        _check(lib().kpp_sched_mlp_loss_grad(self.h, n, _ptr(x), x.shape[1], _ptr(y),
                                             _ptr(self._loss), _stream(x.device)))
        return self._loss

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        _check(lib().kpp_sched_mlp_adam(self.h, lr, beta1, beta2, eps, _stream(self.dev)))

    def features(self, nvar, var, temp, cfactor, sun, tstart, tend=None, dt=0.0,
                 out: Optional[torch.Tensor] = None, col0: int = 0) -> torch.Tensor:
        """Features of the cells into columns col0.. of out (BF16 [nin][ld])."""
        n, ld = var.shape[1], var.shape[1]
        if out is None:
            out = torch.empty(self.nin, n, dtype=torch.bfloat16, device=var.device)
        if out.dtype != torch.bfloat16 or not out.is_contiguous() or col0 + n > out.shape[1]:
            raise SchedError("features: out must be a contiguous bfloat16 [nin][>= col0 + n]")
        _check(lib().kpp_sched_features(self.h, n, ld, nvar, _ptr(var), _ptr(temp),
                                        _ptr(cfactor), _ptr(sun), _ptr(tstart), _ptr(tend),
                                        float(dt), _vp(out.data_ptr() + 2 * col0),
                                        out.shape[1], _stream(var.device)))
        return out


def gather_columns(src: torch.Tensor, idx: torch.Tensor, dst: torch.Tensor):
    _check(lib().kpp_sched_gather_columns(src.shape[0], idx.numel(), _ptr(idx), _ptr(src),
                                          src.shape[1], _ptr(dst), dst.shape[1],
                                          _stream(src.device)))


@dataclass
class LearnedScheduler:
    """A trained network with its scaling and the plan settings."""
    mlp: Mlp
    nvar: int
    in_mu: np.ndarray
    in_sd: np.ndarray
    out_mu: np.ndarray
    out_sd: np.ndarray
    hmin: float = CANDIDATES[0]
    hmax: float = CANDIDATES[-1]
    nbins: int = 1024
    lnn_lo: float = 0.0
    lnn_hi: float = 6.0
    meta: dict = field(default_factory=dict)

    def plan(self, var, temp, tstart, cfactor=None, sun=None, tend=None, dt=0.0,
             hstart: Optional[torch.Tensor] = None, order: Optional[torch.Tensor] = None,
             pred: Optional[torch.Tensor] = None):
        """Per-cell Hstart (float64) and the work-queue order (int32) for one
        chemistry step of the cells; asynchronous."""
        n, ld = var.shape[1], var.shape[1]
        dev = var.device
        if hstart is None:
            hstart = torch.empty(n, dtype=torch.float64, device=dev)
        if order is None:
            order = torch.empty(n, dtype=torch.int32, device=dev)
        _check(lib().kpp_sched_plan(self.mlp.h, n, ld, self.nvar, _ptr(var), _ptr(temp),
                                    _ptr(cfactor), _ptr(sun), _ptr(tstart), _ptr(tend),
                                    float(dt), self.hmin, self.hmax, self.nbins, self.lnn_lo,
                                    self.lnn_hi, _ptr(hstart), _ptr(order), _ptr(pred),
                                    _stream(dev)))
        return hstart, order

    def save(self, path: Path):
        np.savez_compressed(
            path, params=self.mlp.params(), in_mu=self.in_mu, in_sd=self.in_sd,
            out_mu=self.out_mu, out_sd=self.out_sd,
            shape=np.array([self.mlp.nin, self.mlp.width, self.mlp.nhidden, self.mlp.nout]),
            plan=np.array([self.hmin, self.hmax, self.nbins, self.lnn_lo, self.lnn_hi]),
            meta=np.array(repr(self.meta)))

    @classmethod
    def load(cls, path: Path, nvar: int) -> "LearnedScheduler":
        z = np.load(path, allow_pickle=False)
        nin, width, nhidden, nout = (int(v) for v in z["shape"])
        if nin != nvar + 4:
            raise SchedError(f"{path}: network has {nin} inputs, mechanism needs {nvar + 4}")
        mlp = Mlp(nin, width, nhidden, nout)
        mlp.set_params(z["params"])
        mlp.set_scaling(z["in_mu"], z["in_sd"], z["out_mu"], z["out_sd"])
        hmin, hmax, nbins, lo, hi = z["plan"]
        return cls(mlp, nvar, z["in_mu"], z["in_sd"], z["out_mu"], z["out_sd"], float(hmin),
                   float(hmax), int(nbins), float(lo), float(hi), {"source": str(path)})


# ---------------------------------------------------------------- training
def log_tuples(mech, wl, candidates: Sequence[float] = CANDIDATES, chunk: int = 1 << 20,
               verbose: bool = True):
    """Integrates every cell of the workload once per candidate Hstart with
    the plain GPU integrator; returns (nstp [ncand][ncells], ierr_ok [ncells])."""
    dev = torch.device("cuda", torch.cuda.current_device())
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    n = wl.ncells
    nstp = np.zeros((len(candidates), n), dtype=np.int32)
    ok = np.ones(n, dtype=bool)
    atol, rtol = D(wl.atol), D(wl.rtol)
    for sub in _chunks(n, chunk):
        k = sub.stop - sub.start
        fix, temp = D(wl.fix[:, sub]), D(wl.temp[sub])
        cf = D(wl.cfactor[sub]) if wl.cfactor is not None else None
        sun = D(wl.sun[sub]) if wl.sun is not None else None
        t0, t1 = (D(x[sub]) for x in wl.step_bounds(0))
        for j, h in enumerate(candidates):
            t = time.time()
            var = D(wl.var[:, sub])
            hs = torch.full((k,), float(h), dtype=torch.float64, device=dev)
            r = mech.rosenbrock(var, fix, temp, t0, t1, atol, rtol, wl.ipar, wl.rpar, cfactor=cf,
                                sun=sun, hstart=hs)
            nstp[j, sub] = r.istatus[2].cpu().numpy()
            ok[sub] &= (r.ierr == 1).cpu().numpy()
            if verbose:
                print(f"  tuples cells {sub.start}+{k} hstart {h:.1e}: mean steps "
                      f"{nstp[j, sub].mean():.2f} ({time.time() - t:.1f} s)", flush=True)
    return nstp, ok


def targets(nstp: np.ndarray, ok: np.ndarray, candidates: Sequence[float] = CANDIDATES):
    """(log10 Hstart, ln Nstp) per cell: the candidate with the fewest steps
    (the smallest such candidate on ties) and its step count."""
    best = np.argmin(nstp, axis=0)
    cols = np.arange(nstp.shape[1])
    y0 = np.log10(np.asarray(candidates))[best]
    y1 = np.log(np.maximum(nstp[best, cols], 1))
    return np.stack([y0, y1], axis=1), ok


def init_params(nin: int, width: int, nhidden: int, nout: int, seed: int) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for every weight and bias, in the
    parameter layout of include/kpp_sched.h."""
    rng = np.random.default_rng(seed)
    parts = []
    for li in range(nhidden + 1):
        fi = nin if li == 0 else width
        fo = width if li < nhidden else nout
        a = 1.0 / math.sqrt(fi)
        parts += [rng.uniform(-a, a, fo * fi), rng.uniform(-a, a, fo)]
    return np.concatenate(parts).astype(np.float32)


def _chunks(n: int, chunk: int):
    for c0 in range(0, n, chunk):
        yield slice(c0, min(n, c0 + chunk))


def train(wl, nstp: np.ndarray, ok: np.ndarray, epochs: int = 24, batch: int = 8192,
          lr: float = 1e-3, seed: int = 1, holdout: float = 1.0 / 16,
          candidates: Sequence[float] = CANDIDATES, verbose: bool = True) -> LearnedScheduler:
    """Fits the network to the logged tuples with the library's kernels
    (minibatch gather, forward, MSE, backward, Adam; cosine learning rate)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    nvar, n = wl.var.shape[0], wl.ncells
    nin = nvar + 4
    y, ok = targets(nstp, ok, candidates)
    # standardisation statistics of the features (float64, chunked)
    s1 = np.zeros(nin)
    s2 = np.zeros(nin)
    for sub in _chunks(n, 1 << 20):
        f = host_features(wl.var[:, sub], wl.temp[sub],
                          None if wl.cfactor is None else wl.cfactor[sub],
                          None if wl.sun is None else wl.sun[sub], wl.dt)
        s1 += f.sum(axis=1)
        s2 += (f * f).sum(axis=1)
    in_mu = s1 / n
    in_sd = np.sqrt(np.maximum(s2 / n - in_mu ** 2, 0.0))
    in_sd = np.where(in_sd > 1e-6, in_sd, 1.0)
    yo = y[ok]
    out_mu, out_sd = yo.mean(axis=0), np.maximum(yo.std(axis=0), 1e-6)

    mlp = Mlp(nin, max_batch=batch)
    mlp.set_params(init_params(nin, mlp.width, mlp.nhidden, mlp.nout, seed))
    mlp.set_scaling(in_mu, in_sd, out_mu, out_sd)
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    X = torch.empty(nin, n, dtype=torch.bfloat16, device=dev)
    for sub in _chunks(n, 1 << 20):
        mlp.features(nvar, D(wl.var[:, sub]), D(wl.temp[sub]),
                     None if wl.cfactor is None else D(wl.cfactor[sub]),
                     None if wl.sun is None else D(wl.sun[sub]), D(wl.tstart[sub]),
                     dt=wl.dt, out=X, col0=sub.start)
    Y = D(((y - out_mu) / out_sd).astype(np.float32))

    rng = np.random.default_rng(seed)
    cells = rng.permutation(np.nonzero(ok)[0]).astype(np.int32)
    nval = max(int(len(cells) * holdout), 1)
    val, tr = D(cells[:nval]), D(cells[nval:])
    Xb = torch.empty(nin, batch, dtype=torch.bfloat16, device=dev)
    steps_per_epoch = len(tr) // batch
    total = epochs * steps_per_epoch
    history = []
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    t_start = time.time()
    step = 0
    for ep in range(epochs):
        perm = tr[torch.randperm(len(tr), device=dev, generator=gen)]
        acc = torch.zeros(1, dtype=torch.float32, device=dev)
        for b in range(steps_per_epoch):
            idx = perm[b * batch:(b + 1) * batch]
            gather_columns(X, idx, Xb)
            acc += mlp.loss_grad(Xb, Y.index_select(0, idx))
            lr_t = lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * step / max(total, 1))))
            mlp.adam(lr_t)
            step += 1
        train_loss = float(acc.item()) / max(steps_per_epoch, 1)
        history.append(train_loss)
        if verbose:
            print(f"  epoch {ep + 1}/{epochs}: train mse {train_loss:.4f} "
                  f"({time.time() - t_start:.1f} s)", flush=True)
    train_s = time.time() - t_start
    # held-out fit, de-standardised
    Xv = torch.empty(nin, nval, dtype=torch.bfloat16, device=dev)
    gather_columns(X, val, Xv)
    pv = mlp.forward(Xv, nval).cpu().numpy().astype(np.float64) * out_sd + out_mu
    yv = y[cells[:nval]]
    r2 = [float(1.0 - ((pv[:, j] - yv[:, j]) ** 2).mean() / max(yv[:, j].var(), 1e-30))
          for j in range(2)]
    lnn = np.log(np.maximum(nstp, 1))
    meta = {"tuples": int(n), "trained_on": int(len(tr)), "held_out": int(nval),
            "epochs": epochs, "batch": batch, "lr": lr, "train_seconds": round(train_s, 2),
            "final_train_mse": history[-1] if history else None,
            "heldout_r2_log10_hstart": r2[0], "heldout_r2_ln_nstp": r2[1],
            "candidates": list(candidates), "workload": wl.name}
    return LearnedScheduler(mlp, nvar, in_mu.astype(np.float32), in_sd.astype(np.float32),
                            out_mu.astype(np.float32), out_sd.astype(np.float32),
                            hmin=float(min(candidates)), hmax=float(max(candidates)), nbins=1024,
                            lnn_lo=float(lnn.min()) - 0.25, lnn_hi=float(lnn.max()) + 0.25,
                            meta=meta)
