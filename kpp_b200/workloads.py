"""Seeded synthetic grid-cell batches for the benchmark and the tests.

The reference measures on no public dataset; these batches stand in for a
host model's grid, with the shapes, sizes and value distributions of the
benchmark configurations:

  small_strato  (models/small_strato.def): .def concentrations times
      log-uniform factors in [0.5, 2] per species and cell; TEMP = 270 K;
      each cell's start time uniform over 24 h after 12:00 (the sun follows
      Update_SUN through TIME); Rodas3, RTOL 1e-3, ATOL 1.0 (scalar);
      chemistry step 1200 s, 72 steps.
  saprc99       (models/saprc99.def): concentrations log-normal around the
      .def mixing ratios (sigma = 1 in ln units), floored at 1e-20 molec/cm3;
      T uniform 220-310 K; p uniform 200-1013 hPa gives M = p/(k_B T),
      AIR = M, O2 = 0.2095 M, CFACTOR = M/1e6 (ppm -> molec/cm3, used by the
      FALL/EP2/EP3 rate laws) and the other fixed species from their .def
      mixing ratios; a solar zenith angle per cell sets SUN = cos(SZA) by
      day and 0 beyond 90 degrees (SUN is then constant over the step);
      Rodas3, RTOL 1e-3, ATOL 1e-2 (scalar), chemistry step 600 s.
      sza = "uniform95": SZA uniform in 0-95 degrees.
      sza = "classes":   40 % day (0-85), 40 % night (95-180), 20 % within
                         5 degrees of the terminator (85-95).

Arrays are numpy, in the C ABI layout ([rows, ncells], cell index fastest).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .controls import make_controls

SEED_EVAL = 20261203
SEED_TRAIN = 20261204
K_BOLTZMANN = 1.380649e-23  # J/K


@dataclass
class Workload:
    name: str
    mech: str
    ncells: int
    var: np.ndarray            # [NVAR, n]
    fix: np.ndarray            # [NFIX, n]
    temp: np.ndarray           # [n]
    cfactor: Optional[np.ndarray]
    sun: Optional[np.ndarray]
    tstart: np.ndarray         # [n] start of the first chemistry step
    dt: float
    nsteps: int
    atol: np.ndarray
    rtol: np.ndarray
    ipar: List[int]
    rpar: List[float]
    meta: dict = field(default_factory=dict)

    def step_bounds(self, k: int):
        t0 = self.tstart + k * self.dt
        return t0, t0 + self.dt

    def driver_bounds(self, k: int):
        """Bounds of call k of the reference driver loop, TIME += DT
        (drv/general.c:59-76): the times kpp_b200_rosenbrock_chain uses."""
        t0 = self.tstart.copy()
        for _ in range(k):
            t0 = t0 + self.dt
        return t0, t0 + self.dt

    def subset(self, n: int) -> "Workload":
        """The first n cells (same values, same per-cell streams)."""
        sl = slice(0, n)
        opt = lambda a: None if a is None else np.ascontiguousarray(a[..., sl])
        return Workload(self.name, self.mech, n, np.ascontiguousarray(self.var[:, sl]),
                        np.ascontiguousarray(self.fix[:, sl]), self.temp[sl].copy(),
                        opt(self.cfactor), opt(self.sun), self.tstart[sl].copy(), self.dt,
                        self.nsteps, self.atol, self.rtol, list(self.ipar), list(self.rpar),
                        dict(self.meta))


def small_strato(c_default: np.ndarray, nvar: int, ncells: int, seed: int = SEED_EVAL,
                 nsteps: int = 72, method: str = "rodas3") -> Workload:
    """Config 1.  c_default: C[NSPEC] after the mechanism's Initialize()."""
    rng = np.random.default_rng(seed)
    nfix = c_default.size - nvar
    fac = np.exp(rng.uniform(np.log(0.5), np.log(2.0), size=(nvar, ncells)))
    var = np.ascontiguousarray(c_default[:nvar, None] * fac)
    fix = np.ascontiguousarray(np.repeat(c_default[nvar:, None], ncells, axis=1).reshape(nfix, ncells))
    tstart = 12 * 3600.0 + rng.uniform(0.0, 86400.0, size=ncells)
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    return Workload("small_strato_rodas3", "small_strato", ncells, var, fix,
                    np.full(ncells, 270.0), None, None, tstart, 1200.0, nsteps,
                    np.array([1.0]), np.array([1e-3]), ipar, rpar)


def _sza_sample(rng, n: int, mode: str) -> np.ndarray:
    if mode == "uniform95":
        return rng.uniform(0.0, 95.0, size=n)
    if mode == "classes":
        u = rng.uniform(size=n)
        day = rng.uniform(0.0, 85.0, size=n)
        night = rng.uniform(95.0, 180.0, size=n)
        term = rng.uniform(85.0, 95.0, size=n)
        return np.where(u < 0.4, day, np.where(u < 0.8, night, term))
    raise ValueError(mode)


def saprc99(c_default: np.ndarray, cfactor_default: float, species: List[str], nvar: int,
            ncells: int, seed: int = SEED_EVAL, sza: str = "uniform95", nsteps: int = 1,
            method: str = "rodas3") -> Workload:
    """Configs 2, 3 and 5.  c_default: C[NSPEC] after Initialize(); species:
    names in the mechanism's order (variables first)."""
    rng = np.random.default_rng(seed)
    nspec = c_default.size
    ppm = c_default / cfactor_default
    temp = rng.uniform(220.0, 310.0, size=ncells)
    p_hpa = rng.uniform(200.0, 1013.0, size=ncells)
    m = p_hpa * 100.0 / (K_BOLTZMANN * temp) * 1e-6   # molec/cm3
    cfactor = m / 1e6
    logn = rng.standard_normal(size=(nvar, ncells))
    var = np.maximum(ppm[:nvar, None] * cfactor[None, :] * np.exp(logn), 1e-20)
    fix = ppm[nvar:, None] * cfactor[None, :]
    names = [s.upper() for s in species[nvar:nspec]]
    if "AIR" in names:
        fix[names.index("AIR")] = m
    if "O2" in names:
        fix[names.index("O2")] = 0.2095 * m
    angle = _sza_sample(rng, ncells, sza)
    sun = np.where(angle < 90.0, np.cos(np.deg2rad(angle)), 0.0)
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    return Workload(f"saprc99_{sza}", "saprc99", ncells, np.ascontiguousarray(var),
                    np.ascontiguousarray(fix), temp, cfactor, sun,
                    np.full(ncells, 12 * 3600.0), 600.0, nsteps, np.array([1e-2]),
                    np.array([1e-3]), ipar, rpar, meta={"sza": angle, "pressure_hpa": p_hpa})


# Initial mixing ratios of the MCM example driver (examples/mcm/driver_mcm.f90):
# the species it sets, as fractions of M; every other species starts at zero.
MCM_DRIVER_MIXING_RATIOS = {"O3": 3.0e-08, "NO2": 1.0e-10, "CH4": 1.8e-06, "C5H8": 1.0e-09}


def mcm_isoprene(species: List[str], nvar: int, ncells: int, seed: int = SEED_EVAL,
                 nsteps: int = 1, method: str = "rodas4") -> Workload:
    """Config 4: log-normal concentrations (sigma 1, ln units) around the
    example driver's initial mixing ratios times M, every other species at
    the 1e-20 molec/cm3 floor; T uniform 250-310 K, p uniform 200-1013 hPa
    (M = p / kT, the mechanism's CFACTOR), solar zenith angle uniform 0-90
    degrees (SUN = its cosine); Rodas4, RTOL 1e-3, ATOL 1e-2, 300 s steps."""
    rng = np.random.default_rng(seed)
    temp = rng.uniform(250.0, 310.0, size=ncells)
    p_hpa = rng.uniform(200.0, 1013.0, size=ncells)
    m = p_hpa * 100.0 / (K_BOLTZMANN * temp) * 1e-6   # molec/cm3
    frac = np.zeros(nvar)
    for name, x in MCM_DRIVER_MIXING_RATIOS.items():
        frac[[s.upper() for s in species[:nvar]].index(name)] = x
    logn = rng.standard_normal(size=(nvar, ncells))
    var = np.maximum(frac[:, None] * m[None, :] * np.exp(logn), 1e-20)
    angle = rng.uniform(0.0, 90.0, size=ncells)
    sun = np.cos(np.deg2rad(angle))
    ipar, rpar = make_controls(method=method, scalar_tol=True)
    return Workload("mcm_isoprene", "mcm_isoprene", ncells, np.ascontiguousarray(var),
                    np.zeros((0, ncells)), temp, m, sun, np.full(ncells, 12 * 3600.0), 300.0,
                    nsteps, np.array([1e-2]), np.array([1e-3]), ipar, rpar,
                    meta={"sza": angle, "pressure_hpa": p_hpa})


def for_mechanism(mech, name: str, ncells: int, seed: int = SEED_EVAL, **kw) -> Workload:
    """Workload `name` for a loaded kpp_b200.Mechanism (or anything exposing
    initial_values(), species and nvar)."""
    c, cf = mech.initial_values()
    c = np.asarray(c, dtype=np.float64)
    if name == "small_strato":
        return small_strato(c, mech.nvar, ncells, seed, **kw)
    if name.startswith("saprc99"):
        sza = "classes" if name.endswith("classes") else "uniform95"
        return saprc99(c, cf, list(mech.species), mech.nvar, ncells, seed, sza=sza, **kw)
    if name == "mcm_isoprene":
        return mcm_isoprene(list(mech.species), mech.nvar, ncells, seed, **kw)
    raise ValueError(name)
