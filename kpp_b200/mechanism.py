"""Python host layer over the C ABI of include/kpp_b200.h.

A `Mechanism` wraps one mechanism library (libkpp_b200_<mech>.so) through
ctypes.  Device arrays are torch CUDA tensors of float64/int32 in the ABI's
layout: [rows, ld] with the cell index fastest (row-major, contiguous), so the
pointer of tensor[i, c] is var + i*ld + c exactly as the ABI expects.

`Mechanism.integrate` is the batched counterpart of the generated C
`INTEGRATE(TIN, TOUT)` (int/rosenbrock.c:94-133): it calls the batched
Rosenbrock for every cell with the caller's controls and returns the warm
start (Hexit) for the next call, as INTEGRATE keeps STEPMIN = RPAR[11].

There is no CPU fallback: constructing a Mechanism fails when its library is
missing, and the integration entry points require CUDA tensors.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path
from typing import Optional, Sequence

import torch

from . import controls as _controls

LIB_DIR = Path(__file__).resolve().parent / "lib"

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_double_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

KPP_B200_OK = 0


class KppError(RuntimeError):
    pass


@dataclass
class RosenbrockResult:
    """Per-cell outputs: IERR, ISTATUS (IPAR[10..17]) and RSTATUS (Texit, Hexit)."""
    ierr: torch.Tensor      # [ncells] int32
    istatus: torch.Tensor   # [8, ncells] int32: Nfun Njac Nstp Nacc Nrej Ndec Nsol Nsng
    rstatus: torch.Tensor   # [2, ncells] float64: Texit, Hexit

    @property
    def hexit(self) -> torch.Tensor:
        return self.rstatus[1]


def library_path(name: str) -> Path:
    return LIB_DIR / f"libkpp_b200_{name}.so"


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else _vp(t.data_ptr())


class Mechanism:
    """One compiled mechanism: its sizes, species, sparsity and entry points."""

    def __init__(self, name: str, path: Optional[Path] = None):
        path = Path(path) if path else library_path(name)
        if not path.exists():
            raise KppError(f"kpp_b200 library for mechanism {name!r} not found at {path}; "
                           f"build it with `python -m kpp_b200.build {name}`")
        self.path = path
        self.lib = ctypes.CDLL(str(path))
        self._declare()
        dims = (ctypes.c_int * 6)()
        self._check(self.lib.kpp_b200_dims(dims))
        self.nvar, self.nfix, self.nspec, self.nreact, self.lu_nonzero, self.nonzero = list(dims)
        self.name = self.lib.kpp_b200_mechanism_name().decode()
        self.species = [self.lib.kpp_b200_species_name(i).decode() for i in range(self.nspec)]

    # -- ctypes prototypes -------------------------------------------------
    def _declare(self):
        L = self.lib
        L.kpp_b200_dims.argtypes = [_c_int_p]
        L.kpp_b200_mechanism_name.restype = ctypes.c_char_p
        L.kpp_b200_species_name.argtypes = [ctypes.c_int]
        L.kpp_b200_species_name.restype = ctypes.c_char_p
        L.kpp_b200_initial_values.argtypes = [_c_double_p, _c_double_p]
        L.kpp_b200_lu_pattern.argtypes = [_c_int_p] * 4
        L.kpp_b200_last_error.restype = ctypes.c_char_p
        L.kpp_b200_workspace_bytes.argtypes = [ctypes.c_int]
        L.kpp_b200_workspace_bytes.restype = ctypes.c_size_t
        ros = [ctypes.c_int, ctypes.c_int] + [_vp] * 9 + [_c_int_p, _c_double_p, _vp, _vp, _vp, _vp]
        L.kpp_b200_rosenbrock.argtypes = ros + [_vp]
        L.kpp_b200_rosenbrock_ws.argtypes = ros + [_vp, ctypes.c_size_t, _vp]
        L.kpp_b200_rosenbrock_host.argtypes = ros + [ctypes.c_int]
        L.kpp_b200_fun_jac.argtypes = [ctypes.c_int, ctypes.c_int] + [_vp] * 5 + [ctypes.c_double] + [_vp] * 4
        L.kpp_b200_decomp_solve.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]
        L.kpp_b200_jac_vec.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int,
                                       _vp]
        L.kpp_b200_solve_tr.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]
        L.kpp_b200_set_kernel.argtypes = [ctypes.c_int]
        L.kpp_b200_set_blocks_per_sm.argtypes = [ctypes.c_int]
        L.kpp_b200_set_auto_warp_cells.argtypes = [ctypes.c_int]
        L.kpp_b200_set_queue_lanes.argtypes = [ctypes.c_int]
        L.kpp_b200_sdirk.argtypes = ([ctypes.c_int, ctypes.c_int] + [_vp] * 9
                                     + [ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_double)] + [_vp] * 4)
        L.kpp_b200_runge_kutta.argtypes = L.kpp_b200_sdirk.argtypes
        L.kpp_b200_sdirk_host.argtypes = L.kpp_b200_sdirk.argtypes[:-1] + [ctypes.c_int]
        L.kpp_b200_runge_kutta_host.argtypes = L.kpp_b200_sdirk_host.argtypes
        L.kpp_b200_rosenbrock_adj_work_bytes.argtypes = [ctypes.c_int] * 4
        L.kpp_b200_rosenbrock_adj_work_bytes.restype = ctypes.c_size_t
        L.kpp_b200_rosenbrock_adj.argtypes = (
            [ctypes.c_int, ctypes.c_int] + [_vp] * 9 + [ctypes.c_int, _vp]
            + [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_int, _vp,
               ctypes.c_size_t] + [_vp] * 4)
        L.kpp_b200_user_species.argtypes = [_vp, _vp]
        L.kpp_b200_shuffle_user2kpp.argtypes = [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                _vp, _vp]
        L.kpp_b200_shuffle_kpp2user.argtypes = [ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                _vp, _vp]
        L.kpp_b200_rosenbrock_chain.argtypes = (
            [ctypes.c_int, ctypes.c_int] + [_vp] * 6 + [ctypes.c_double, ctypes.c_int]
            + [_vp] * 2 + [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
            + [_vp] * 6)

    def _check(self, rc: int):
        if rc != KPP_B200_OK:
            raise KppError(f"kpp_b200 error {rc}: {self.lib.kpp_b200_last_error().decode()}")

    # -- mechanism description --------------------------------------------
    def initial_values(self):
        """(C[NSPEC] after Initialize(), CFACTOR)."""
        c = (ctypes.c_double * self.nspec)()
        cf = ctypes.c_double()
        self._check(self.lib.kpp_b200_initial_values(c, ctypes.byref(cf)))
        return list(c), cf.value

    def lu_pattern(self):
        n, nz = self.nvar, self.lu_nonzero
        irow, icol = (ctypes.c_int * nz)(), (ctypes.c_int * nz)()
        crow, diag = (ctypes.c_int * (n + 1))(), (ctypes.c_int * (n + 1))()
        self._check(self.lib.kpp_b200_lu_pattern(irow, icol, crow, diag))
        return list(irow), list(icol), list(crow), list(diag)

    def index(self, species: str) -> int:
        return self.species.index(species)

    def set_kernel(self, which: str):
        """'auto', 'thread' (one thread per cell) or 'warp' (one warp per cell,
        work set in shared memory); both give bit-identical results."""
        self._check(self.lib.kpp_b200_set_kernel({"auto": 0, "thread": 1, "warp": 2}[which]))

    def set_auto_warp_cells(self, ncells: int):
        """Launches of at most `ncells` cells run on the warp-per-cell kernel
        under the automatic choice (when it supports them); 0: never."""
        self._check(self.lib.kpp_b200_set_auto_warp_cells(int(ncells)))

    def auto_warp_cells(self) -> int:
        return int(self.lib.kpp_b200_get_auto_warp_cells())

    def set_queue_lanes(self, per_lane: bool):
        """Work-queue granularity of rosenbrock_chain: each lane takes one
        cell at a time and the lanes' cells advance one step attempt at a
        time together (True, the default), or each warp takes 32 cells
        (False).  Results are the same bit for bit."""
        self._check(self.lib.kpp_b200_set_queue_lanes(1 if per_lane else 0))

    def queue_lanes(self) -> bool:
        return bool(self.lib.kpp_b200_get_queue_lanes())

    def user_species(self):
        """kpp_index[k] of every user species k (declaration order of the
        variable species; -1: not in the mechanism), as a list."""
        n = ctypes.c_int()
        self._check(self.lib.kpp_b200_user_species(ctypes.byref(n), None))
        idx = (ctypes.c_int * max(n.value, 1))()
        self._check(self.lib.kpp_b200_user_species(None, idx))
        return list(idx)[:n.value]

    def shuffle_user2kpp(self, v_user: torch.Tensor, var: torch.Tensor,
                         stream: Optional[torch.cuda.Stream] = None):
        """var rows of the mapped user species from v_user ([nuser][ld_user])."""
        self._dev(v_user, torch.float64, "v_user")
        self._dev(var, torch.float64, "var")
        n = var.shape[1]
        s = stream if stream is not None else torch.cuda.current_stream(var.device)
        self._check(self.lib.kpp_b200_shuffle_user2kpp(n, v_user.shape[1], _ptr(v_user),
                                                       var.shape[1], _ptr(var),
                                                       _vp(s.cuda_stream)))

    def shuffle_kpp2user(self, var: torch.Tensor, v_user: torch.Tensor,
                         stream: Optional[torch.cuda.Stream] = None):
        self._dev(v_user, torch.float64, "v_user")
        self._dev(var, torch.float64, "var")
        n = var.shape[1]
        s = stream if stream is not None else torch.cuda.current_stream(var.device)
        self._check(self.lib.kpp_b200_shuffle_kpp2user(n, var.shape[1], _ptr(var),
                                                       v_user.shape[1], _ptr(v_user),
                                                       _vp(s.cuda_stream)))

    def set_blocks_per_sm(self, blocks: int):
        """Resident 128-thread blocks per SM of the thread-per-cell launches
        (0: as many as fit); the results do not depend on it."""
        self._check(self.lib.kpp_b200_set_blocks_per_sm(int(blocks)))

    def blocks_per_sm(self) -> int:
        return self.lib.kpp_b200_get_blocks_per_sm()

    def kernel(self) -> str:
        return {1: "thread", 2: "warp"}[self.lib.kpp_b200_get_kernel()]

    def workspace_bytes(self, ncells: int) -> int:
        return int(self.lib.kpp_b200_workspace_bytes(ncells))

    # -- batched entry points ---------------------------------------------
    @staticmethod
    def _dev(t, dtype, name):
        if t is None:
            return None
        if not (isinstance(t, torch.Tensor) and t.is_cuda):
            raise KppError(f"{name} must be a CUDA tensor (the path has no CPU fallback)")
        if t.dtype != dtype or not t.is_contiguous():
            raise KppError(f"{name} must be a contiguous {dtype} tensor")
        return t

    def _shapes(self, ld: int, n: int, rows=(), cols=(), device=None, tol=None, vector_tol=False):
        """Shapes the C ABI reads or writes, checked before the call so that a
        wrong shape is a KppError rather than an out-of-bounds device access.
        rows: (tensor, name, nrows) that must be [nrows, ld] (the ABI's leading
        dimension is ld for every batched 2-D array); cols: (tensor, name) 1-D
        arrays indexed by cell, at least n entries; tol: (atol, rtol), NVAR
        entries with vector tolerances, else 1; every tensor on `device`."""
        if not 0 <= n <= ld:
            raise KppError(f"ncells must be in [0, ld]: ncells={n}, ld={ld}")
        allt = []
        for t, nm, nr in rows:
            if t is None:
                continue
            if t.dim() != 2 or t.shape[0] != nr or t.shape[1] != ld:
                raise KppError(f"{nm} must have shape [{nr}, {ld}], got {list(t.shape)}")
            allt.append((t, nm))
        for t, nm in cols:
            if t is None:
                continue
            if t.dim() != 1 or t.shape[0] < n:
                raise KppError(f"{nm} must be 1-D with at least {n} entries, got {list(t.shape)}")
            allt.append((t, nm))
        if tol is not None:
            need = self.nvar if vector_tol else 1
            for t, nm in zip(tol, ("atol", "rtol")):
                if t is None or t.numel() < need:
                    raise KppError(f"{nm} needs at least {need} entries")
                allt.append((t, nm))
        if device is not None:
            for t, nm in allt:
                if t.device != device:
                    raise KppError(f"{nm} is on {t.device}, expected {device}")

    def _outputs(self, out, ld, rstatus_rows, device):
        if out is not None:
            self._shapes(ld, ld, rows=((out.istatus, "out.istatus", 8),
                                       (out.rstatus, "out.rstatus", rstatus_rows)),
                         cols=((out.ierr, "out.ierr"),), device=device)
            if out.ierr.shape[0] != ld:
                raise KppError(f"out.ierr must have {ld} entries")

    def rosenbrock(self, var: torch.Tensor, fix: torch.Tensor, temp: torch.Tensor,
                   tstart: torch.Tensor, tend: torch.Tensor, atol: torch.Tensor,
                   rtol: torch.Tensor, ipar: Sequence[int], rpar: Sequence[float],
                   cfactor: Optional[torch.Tensor] = None, sun: Optional[torch.Tensor] = None,
                   hstart: Optional[torch.Tensor] = None, ncells: Optional[int] = None,
                   out: Optional[RosenbrockResult] = None,
                   workspace: Optional[torch.Tensor] = None,
                   stream: Optional[torch.cuda.Stream] = None) -> RosenbrockResult:
        """Batched Rosenbrock (kpp_b200_rosenbrock).  var [NVAR, ld] is updated
        in place; returns IERR/ISTATUS/RSTATUS.  Asynchronous on `stream`."""
        f64, i32 = torch.float64, torch.int32
        self._dev(var, f64, "var")
        ld = var.shape[1]
        n = ld if ncells is None else ncells
        for t, nm in ((fix, "fix"), (temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                      (atol, "atol"), (rtol, "rtol"), (cfactor, "cfactor"), (sun, "sun"),
                      (hstart, "hstart")):
            self._dev(t, f64, nm)
        self._shapes(ld, n, rows=((var, "var", self.nvar), (fix, "fix", self.nfix)),
                     cols=((temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                           (cfactor, "cfactor"), (sun, "sun"), (hstart, "hstart")),
                     device=var.device, tol=(atol, rtol), vector_tol=int(ipar[1]) == 0)
        self._outputs(out, ld, 2, var.device)
        if out is None:
            out = RosenbrockResult(ierr=torch.empty(ld, dtype=i32, device=var.device),
                                   istatus=torch.empty(8, ld, dtype=i32, device=var.device),
                                   rstatus=torch.empty(2, ld, dtype=f64, device=var.device))
        ip = (ctypes.c_int * 20)(*[int(x) for x in ipar])
        rp = (ctypes.c_double * 20)(*[float(x) for x in rpar])
        s = stream if stream is not None else torch.cuda.current_stream(var.device)
        args = [n, ld, _ptr(var), _ptr(fix), _ptr(temp), _ptr(cfactor), _ptr(sun),
                _ptr(tstart), _ptr(tend), _ptr(atol), _ptr(rtol), ip, rp, _ptr(hstart),
                _ptr(out.istatus), _ptr(out.rstatus), _ptr(out.ierr)]
        if workspace is not None:
            self._check(self.lib.kpp_b200_rosenbrock_ws(
                *args, _ptr(workspace), workspace.numel() * workspace.element_size(),
                _vp(s.cuda_stream)))
        else:
            self._check(self.lib.kpp_b200_rosenbrock(*args, _vp(s.cuda_stream)))
        return out

    def sdirk(self, var: torch.Tensor, fix: torch.Tensor, temp: torch.Tensor,
              tstart: torch.Tensor, tend: torch.Tensor, atol: torch.Tensor, rtol: torch.Tensor,
              icntrl: Sequence[int], rcntrl: Sequence[float],
              cfactor: Optional[torch.Tensor] = None, sun: Optional[torch.Tensor] = None,
              ncells: Optional[int] = None, out: Optional[RosenbrockResult] = None,
              stream: Optional[torch.cuda.Stream] = None) -> RosenbrockResult:
        """The reference's C SDIRK integrator for every cell (kpp_b200_sdirk):
        ICNTRL / RCNTRL in the C layout; istatus = ISTATUS[1..8], rstatus
        [3, ld] = RSTATUS[1..3] (Texit, Hexit, Hnew); ierr 1 or 0."""
        f64, i32 = torch.float64, torch.int32
        self._dev(var, f64, "var")
        ld = var.shape[1]
        n = ld if ncells is None else ncells
        for t, nm in ((fix, "fix"), (temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                      (atol, "atol"), (rtol, "rtol"), (cfactor, "cfactor"), (sun, "sun")):
            self._dev(t, f64, nm)
        self._shapes(ld, n, rows=((var, "var", self.nvar), (fix, "fix", self.nfix)),
                     cols=((temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                           (cfactor, "cfactor"), (sun, "sun")),
                     device=var.device, tol=(atol, rtol), vector_tol=int(icntrl[1]) == 0)
        self._outputs(out, ld, 3, var.device)
        if out is None:
            out = RosenbrockResult(ierr=torch.empty(ld, dtype=i32, device=var.device),
                                   istatus=torch.empty(8, ld, dtype=i32, device=var.device),
                                   rstatus=torch.empty(3, ld, dtype=f64, device=var.device))
        ic = (ctypes.c_int * 20)(*[int(x) for x in icntrl])
        rc = (ctypes.c_double * 20)(*[float(x) for x in rcntrl])
        s = stream if stream is not None else torch.cuda.current_stream(var.device)
        self._check(self.lib.kpp_b200_sdirk(
            n, ld, _ptr(var), _ptr(fix), _ptr(temp), _ptr(cfactor), _ptr(sun), _ptr(tstart),
            _ptr(tend), _ptr(atol), _ptr(rtol), ic, rc, _ptr(out.istatus), _ptr(out.rstatus),
            _ptr(out.ierr), _vp(s.cuda_stream)))
        return out

    def runge_kutta(self, var: torch.Tensor, fix: torch.Tensor, temp: torch.Tensor,
                    tstart: torch.Tensor, tend: torch.Tensor, atol: torch.Tensor,
                    rtol: torch.Tensor, icntrl: Sequence[int], rcntrl: Sequence[float],
                    cfactor: Optional[torch.Tensor] = None, sun: Optional[torch.Tensor] = None,
                    ncells: Optional[int] = None, out: Optional[RosenbrockResult] = None,
                    stream: Optional[torch.cuda.Stream] = None) -> RosenbrockResult:
        """The reference's C RungeKutta integrator for every cell
        (kpp_b200_runge_kutta): ICNTRL / RCNTRL in the C layout; istatus =
        ISTATUS[0..7], rstatus [3, ld] = RSTATUS[0..2] (Texit, Hacc, Hnew)."""
        f64, i32 = torch.float64, torch.int32
        self._dev(var, f64, "var")
        ld = var.shape[1]
        n = ld if ncells is None else ncells
        for t, nm in ((fix, "fix"), (temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                      (atol, "atol"), (rtol, "rtol"), (cfactor, "cfactor"), (sun, "sun")):
            self._dev(t, f64, nm)
        self._shapes(ld, n, rows=((var, "var", self.nvar), (fix, "fix", self.nfix)),
                     cols=((temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                           (cfactor, "cfactor"), (sun, "sun")),
                     device=var.device, tol=(atol, rtol), vector_tol=int(icntrl[1]) == 0)
        self._outputs(out, ld, 3, var.device)
        if out is None:
            out = RosenbrockResult(ierr=torch.empty(ld, dtype=i32, device=var.device),
                                   istatus=torch.empty(8, ld, dtype=i32, device=var.device),
                                   rstatus=torch.empty(3, ld, dtype=f64, device=var.device))
        ic = (ctypes.c_int * 20)(*[int(x) for x in icntrl])
        rc = (ctypes.c_double * 20)(*[float(x) for x in rcntrl])
        s = stream if stream is not None else torch.cuda.current_stream(var.device)
        self._check(self.lib.kpp_b200_runge_kutta(
            n, ld, _ptr(var), _ptr(fix), _ptr(temp), _ptr(cfactor), _ptr(sun), _ptr(tstart),
            _ptr(tend), _ptr(atol), _ptr(rtol), ic, rc, _ptr(out.istatus), _ptr(out.rstatus),
            _ptr(out.ierr), _vp(s.cuda_stream)))
        return out

    def rosenbrock_adj(self, var: torch.Tensor, fix: torch.Tensor, temp: torch.Tensor,
                       tstart: torch.Tensor, tend: torch.Tensor, atol: torch.Tensor,
                       rtol: torch.Tensor, lam: torch.Tensor, icntrl: Sequence[int],
                       rcntrl: Sequence[float], bufsize: int = 1000,
                       cfactor: Optional[torch.Tensor] = None, sun: Optional[torch.Tensor] = None,
                       ncells: Optional[int] = None, out: Optional[RosenbrockResult] = None,
                       work: Optional[torch.Tensor] = None,
                       stream: Optional[torch.cuda.Stream] = None) -> RosenbrockResult:
        """The reference's Rosenbrock discrete adjoint for every cell
        (kpp_b200_rosenbrock_adj, libraries built on KPP's own generator):
        var and lam [NADJ * NVAR, ld] in place; ICNTRL / RCNTRL in the C
        layout of int/rosenbrock_adj.c; bufsize = trajectory entries per cell
        (the step limit is bufsize - 1); istatus = ISTATUS[1..8], rstatus
        [3, ld] = Texit, Hexit, Hnew.  work: a float64 device buffer of at
        least kpp_b200_rosenbrock_adj_work_bytes bytes, else allocated here.
        Asynchronous."""
        f64, i32 = torch.float64, torch.int32
        self._dev(var, f64, "var")
        self._dev(lam, f64, "lam")
        ld = var.shape[1]
        n = ld if ncells is None else ncells
        for t, nm in ((fix, "fix"), (temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                      (atol, "atol"), (rtol, "rtol"), (cfactor, "cfactor"), (sun, "sun")):
            self._dev(t, f64, nm)
        if lam.dim() != 2 or lam.shape[1] != ld or lam.shape[0] % self.nvar:
            raise KppError(f"lam must have shape [NADJ * {self.nvar}, {ld}], got "
                           f"{list(lam.shape)}")
        nadj = lam.shape[0] // self.nvar
        self._shapes(ld, n, rows=((var, "var", self.nvar), (fix, "fix", self.nfix)),
                     cols=((temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                           (cfactor, "cfactor"), (sun, "sun")),
                     device=var.device, tol=(atol, rtol), vector_tol=int(icntrl[1]) == 0)
        self._outputs(out, ld, 3, var.device)
        if out is None:
            out = RosenbrockResult(ierr=torch.empty(ld, dtype=i32, device=var.device),
                                   istatus=torch.empty(8, ld, dtype=i32, device=var.device),
                                   rstatus=torch.empty(3, ld, dtype=f64, device=var.device))
        nbytes = int(self.lib.kpp_b200_rosenbrock_adj_work_bytes(ld, nadj, int(bufsize),
                                                                 int(icntrl[7])))
        if work is None:
            work = torch.empty(max(nbytes // 8, 1), dtype=f64, device=var.device)
        self._dev(work, f64, "work")
        if work.numel() * 8 < nbytes:
            raise KppError(f"work must hold {nbytes} bytes, has {work.numel() * 8}")
        ic = (ctypes.c_int * 20)(*[int(x) for x in icntrl])
        rc = (ctypes.c_double * 20)(*[float(x) for x in rcntrl])
        s = stream if stream is not None else torch.cuda.current_stream(var.device)
        self._check(self.lib.kpp_b200_rosenbrock_adj(
            n, ld, _ptr(var), _ptr(fix), _ptr(temp), _ptr(cfactor), _ptr(sun), _ptr(tstart),
            _ptr(tend), _ptr(atol), _ptr(rtol), nadj, _ptr(lam), ic, rc, int(bufsize),
            _ptr(work), work.numel() * 8, _ptr(out.istatus), _ptr(out.rstatus), _ptr(out.ierr),
            _vp(s.cuda_stream)))
        out.work = work  # kept alive until the caller drops the result
        return out

    def rosenbrock_chain(self, var: torch.Tensor, fix: torch.Tensor, temp: torch.Tensor,
                         tstart: torch.Tensor, dt: float, ncalls: int, atol: torch.Tensor,
                         rtol: torch.Tensor, ipar: Sequence[int], rpar: Sequence[float],
                         cfactor: Optional[torch.Tensor] = None,
                         sun: Optional[torch.Tensor] = None,
                         hstart: Optional[torch.Tensor] = None,
                         order: Optional[torch.Tensor] = None, ncells: Optional[int] = None,
                         out: Optional[RosenbrockResult] = None,
                         stream: Optional[torch.cuda.Stream] = None) -> RosenbrockResult:
        """The driver loop over INTEGRATE for every cell in one persistent
        launch (kpp_b200_rosenbrock_chain): `ncalls` calls of `dt` seconds
        from tstart, Hstart chained from Hexit, counters summed.  `order`
        (int32 permutation) is the work-queue order.  Asynchronous."""
        f64, i32 = torch.float64, torch.int32
        self._dev(var, f64, "var")
        ld = var.shape[1]
        n = ld if ncells is None else ncells
        for t, nm in ((fix, "fix"), (temp, "temp"), (tstart, "tstart"), (atol, "atol"),
                      (rtol, "rtol"), (cfactor, "cfactor"), (sun, "sun"), (hstart, "hstart")):
            self._dev(t, f64, nm)
        self._dev(order, i32, "order")
        self._shapes(ld, n, rows=((var, "var", self.nvar), (fix, "fix", self.nfix)),
                     cols=((temp, "temp"), (tstart, "tstart"), (cfactor, "cfactor"),
                           (sun, "sun"), (hstart, "hstart"), (order, "order")),
                     device=var.device, tol=(atol, rtol), vector_tol=int(ipar[1]) == 0)
        self._outputs(out, ld, 2, var.device)
        if out is None:
            out = RosenbrockResult(ierr=torch.empty(ld, dtype=i32, device=var.device),
                                   istatus=torch.empty(8, ld, dtype=i32, device=var.device),
                                   rstatus=torch.empty(2, ld, dtype=f64, device=var.device))
        ip = (ctypes.c_int * 20)(*[int(x) for x in ipar])
        rp = (ctypes.c_double * 20)(*[float(x) for x in rpar])
        s = stream if stream is not None else torch.cuda.current_stream(var.device)
        self._check(self.lib.kpp_b200_rosenbrock_chain(
            n, ld, _ptr(var), _ptr(fix), _ptr(temp), _ptr(cfactor), _ptr(sun), _ptr(tstart),
            float(dt), int(ncalls), _ptr(atol), _ptr(rtol), ip, rp, _ptr(hstart), _ptr(order),
            _ptr(out.istatus), _ptr(out.rstatus), _ptr(out.ierr), _vp(s.cuda_stream)))
        return out

    @staticmethod
    def _host(t, dtype, name):
        if t is None:
            return None
        if not isinstance(t, torch.Tensor) or t.is_cuda:
            raise KppError(f"{name} must be a host (CPU) tensor")
        if t.dtype != dtype or not t.is_contiguous():
            raise KppError(f"{name} must be a contiguous {dtype} tensor")
        return t

    def rosenbrock_host(self, var, fix, temp, tstart, tend, atol, rtol, ipar, rpar,
                        cfactor=None, sun=None, hstart=None, ncells=None, out=None,
                        chunk: int = 0) -> RosenbrockResult:
        """Batched Rosenbrock on host tensors (kpp_b200_rosenbrock_host): chunked
        copies overlapped with the integration; synchronous.  Pinned tensors
        give full overlap."""
        f64, i32 = torch.float64, torch.int32
        self._host(var, f64, "var")
        ld = var.shape[1]
        n = ld if ncells is None else ncells
        for t, nm in ((fix, "fix"), (temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                      (atol, "atol"), (rtol, "rtol"), (cfactor, "cfactor"), (sun, "sun"),
                      (hstart, "hstart")):
            self._host(t, f64, nm)
        if out is None:
            pin = torch.cuda.is_available()
            out = RosenbrockResult(ierr=torch.empty(ld, dtype=i32, pin_memory=pin),
                                   istatus=torch.empty(8, ld, dtype=i32, pin_memory=pin),
                                   rstatus=torch.empty(2, ld, dtype=f64, pin_memory=pin))
        ip = (ctypes.c_int * 20)(*[int(x) for x in ipar])
        rp = (ctypes.c_double * 20)(*[float(x) for x in rpar])
        self._check(self.lib.kpp_b200_rosenbrock_host(
            n, ld, _ptr(var), _ptr(fix), _ptr(temp), _ptr(cfactor), _ptr(sun), _ptr(tstart),
            _ptr(tend), _ptr(atol), _ptr(rtol), ip, rp, _ptr(hstart), _ptr(out.istatus),
            _ptr(out.rstatus), _ptr(out.ierr), int(chunk)))
        return out

    def sdirk_host(self, var, fix, temp, tstart, tend, atol, rtol, icntrl, rcntrl,
                   cfactor=None, sun=None, ncells=None, out=None,
                   chunk: int = 0) -> RosenbrockResult:
        """kpp_b200_sdirk on host tensors (kpp_b200_sdirk_host); synchronous."""
        return self._integrator_host(self.lib.kpp_b200_sdirk_host, var, fix, temp, tstart,
                                     tend, atol, rtol, icntrl, rcntrl, cfactor, sun, ncells,
                                     out, chunk)

    def runge_kutta_host(self, var, fix, temp, tstart, tend, atol, rtol, icntrl, rcntrl,
                         cfactor=None, sun=None, ncells=None, out=None,
                         chunk: int = 0) -> RosenbrockResult:
        """kpp_b200_runge_kutta on host tensors (kpp_b200_runge_kutta_host);
        synchronous."""
        return self._integrator_host(self.lib.kpp_b200_runge_kutta_host, var, fix, temp,
                                     tstart, tend, atol, rtol, icntrl, rcntrl, cfactor, sun,
                                     ncells, out, chunk)

    def _integrator_host(self, entry, var, fix, temp, tstart, tend, atol, rtol, icntrl, rcntrl,
                         cfactor, sun, ncells, out, chunk):
        f64, i32 = torch.float64, torch.int32
        self._host(var, f64, "var")
        ld = var.shape[1]
        n = ld if ncells is None else ncells
        for t, nm in ((fix, "fix"), (temp, "temp"), (tstart, "tstart"), (tend, "tend"),
                      (atol, "atol"), (rtol, "rtol"), (cfactor, "cfactor"), (sun, "sun")):
            self._host(t, f64, nm)
        if out is None:
            pin = torch.cuda.is_available()
            out = RosenbrockResult(ierr=torch.empty(ld, dtype=i32, pin_memory=pin),
                                   istatus=torch.empty(8, ld, dtype=i32, pin_memory=pin),
                                   rstatus=torch.empty(3, ld, dtype=f64, pin_memory=pin))
        ic = (ctypes.c_int * 20)(*[int(x) for x in icntrl])
        rc = (ctypes.c_double * 20)(*[float(x) for x in rcntrl])
        self._check(entry(n, ld, _ptr(var), _ptr(fix), _ptr(temp), _ptr(cfactor), _ptr(sun),
                          _ptr(tstart), _ptr(tend), _ptr(atol), _ptr(rtol), ic, rc,
                          _ptr(out.istatus), _ptr(out.rstatus), _ptr(out.ierr), int(chunk)))
        return out

    def fun_jac(self, var, fix, temp, time: float, cfactor=None, sun=None,
                want=("rconst", "vdot", "jvs"), stream=None):
        """Batched Update_RCONST / Fun / Jac_SP at one time (kpp_b200_fun_jac)."""
        f64 = torch.float64
        self._dev(var, f64, "var")
        for t, nm in ((fix, "fix"), (temp, "temp"), (cfactor, "cfactor"), (sun, "sun")):
            self._dev(t, f64, nm)
        ld = var.shape[1]
        dev = var.device
        self._shapes(ld, ld, rows=((var, "var", self.nvar), (fix, "fix", self.nfix)),
                     cols=((temp, "temp"), (cfactor, "cfactor"), (sun, "sun")), device=dev)
        rconst = torch.empty(self.nreact, ld, dtype=f64, device=dev) if "rconst" in want else None
        vdot = torch.empty(self.nvar, ld, dtype=f64, device=dev) if "vdot" in want else None
        jvs = torch.empty(self.lu_nonzero, ld, dtype=f64, device=dev) if "jvs" in want else None
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        self._check(self.lib.kpp_b200_fun_jac(ld, ld, _ptr(var), _ptr(fix), _ptr(temp),
                                              _ptr(cfactor), _ptr(sun), float(time),
                                              _ptr(rconst), _ptr(vdot), _ptr(jvs),
                                              _vp(s.cuda_stream)))
        return rconst, vdot, jvs

    def decomp_solve(self, jvs: torch.Tensor, x: Optional[torch.Tensor] = None, stream=None):
        """In-place batched KppDecomp (+ KppSolve of x); returns ising [ld]."""
        self._dev(jvs, torch.float64, "jvs")
        self._dev(x, torch.float64, "x")
        ld = jvs.shape[1]
        self._shapes(ld, ld, rows=((jvs, "jvs", self.lu_nonzero), (x, "x", self.nvar)),
                     device=jvs.device)
        ising = torch.empty(ld, dtype=torch.int32, device=jvs.device)
        s = stream if stream is not None else torch.cuda.current_stream(jvs.device)
        self._check(self.lib.kpp_b200_decomp_solve(ld, ld, _ptr(jvs), _ptr(x), _ptr(ising),
                                                   _vp(s.cuda_stream)))
        return ising

    def jac_vec(self, jvs: torch.Tensor, uv: torch.Tensor, transposed: bool = False,
                out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        """Batched J uv or J^T uv (kpp_b200_jac_vec; Jac_SP_Vec / JacTR_SP_Vec)
        with jvs [LU_NONZERO, ld] and uv [NVAR, ld]."""
        self._dev(jvs, torch.float64, "jvs")
        self._dev(uv, torch.float64, "uv")
        self._dev(out, torch.float64, "out")
        ld = jvs.shape[1]
        self._shapes(ld, ld, rows=((jvs, "jvs", self.lu_nonzero), (uv, "uv", self.nvar),
                                   (out, "out", self.nvar)), device=jvs.device)
        if out is None:
            out = torch.empty_like(uv)
        s = stream if stream is not None else torch.cuda.current_stream(jvs.device)
        self._check(self.lib.kpp_b200_jac_vec(ld, ld, _ptr(jvs), _ptr(uv), _ptr(out),
                                              1 if transposed else 0, _vp(s.cuda_stream)))
        return out

    def solve_tr(self, jvs: torch.Tensor, x: torch.Tensor, out: Optional[torch.Tensor] = None,
                 stream=None) -> torch.Tensor:
        """Batched solve of (LU)^T xx = x for factorised jvs (kpp_b200_solve_tr;
        KppSolveTR)."""
        self._dev(jvs, torch.float64, "jvs")
        self._dev(x, torch.float64, "x")
        self._dev(out, torch.float64, "out")
        ld = jvs.shape[1]
        self._shapes(ld, ld, rows=((jvs, "jvs", self.lu_nonzero), (x, "x", self.nvar),
                                   (out, "out", self.nvar)), device=jvs.device)
        if out is None:
            out = torch.empty_like(x)
        s = stream if stream is not None else torch.cuda.current_stream(jvs.device)
        self._check(self.lib.kpp_b200_solve_tr(ld, ld, _ptr(jvs), _ptr(x), _ptr(out),
                                               _vp(s.cuda_stream)))
        return out

    # -- INTEGRATE-style driver -------------------------------------------
    def integrate(self, var, fix, temp, tin, tout, atol, rtol, method: str = "rodas3",
                  stepmin=None, cfactor=None, sun=None, **controls) -> RosenbrockResult:
        """One chemistry step for every cell, like the generated INTEGRATE(TIN,
        TOUT): non-autonomous, the given method, starting step `stepmin`
        (per cell, the previous call's Hexit; None = default)."""
        ipar, rpar = _controls.make_controls(method=method, scalar_tol=atol.numel() == 1,
                                             **controls)
        return self.rosenbrock(var, fix, temp, tin, tout, atol, rtol, ipar, rpar,
                               cfactor=cfactor, sun=sun, hstart=stepmin)


_loaded = {}


def load(name: str) -> Mechanism:
    """Load (once per process) the library of mechanism `name`."""
    if name not in _loaded:
        _loaded[name] = Mechanism(name)
    return _loaded[name]
