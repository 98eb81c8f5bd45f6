"""Integrator controls of the C Rosenbrock (IPAR/RPAR) and the F90 layout
(ICNTRL/RCNTRL).

The C ABI takes the controls in the C layout of int/rosenbrock.c:201-254
(the reference path being matched is the C one).  KPP's Fortran integrator
names the same controls ICNTRL/RCNTRL (int/rosenbrock.f90:180-240) with two
entries swapped; `from_fortran` converts.

  C IPAR[0] = ICNTRL(1)  autonomous (1) / time dependent (0)
  C IPAR[1] = ICNTRL(2)  scalar (1) / vector (0) tolerances
  C IPAR[2] = ICNTRL(4)  maximum number of steps (0: 100000)
  C IPAR[3] = ICNTRL(3)  method: 1 Ros2, 2 Ros3, 3 Ros4, 4 Rodas3, 5 Rodas4
  C RPAR[0..6] = RCNTRL(1..7)  Hmin, Hmax, Hstart, FacMin, FacMax, FacRej, FacSafe
  C IPAR[10..17] = ISTATUS(1..8), C RPAR[10..11] = RSTATUS(1..2)
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

METHODS = {"ros2": 1, "ros3": 2, "ros4": 3, "rodas3": 4, "rodas4": 5}

ISTATUS_NAMES = ["Nfun", "Njac", "Nstp", "Nacc", "Nrej", "Ndec", "Nsol", "Nsng"]

IERR_TEXT = {
    1: "success",
    -1: "improper value for maximal no of steps",
    -2: "selected Rosenbrock method not implemented",
    -3: "Hmin/Hmax/Hstart must be positive",
    -4: "FacMin/FacMax/FacRej must be positive",
    -5: "improper tolerance values",
    -6: "no of steps exceeds maximum bound",
    -7: "step size too small (T + H/10 = T) or H < Roundoff",
    -8: "matrix is repeatedly singular",
}


def make_controls(method="rodas3", scalar_tol=True, autonomous=False, max_steps=0,
                  hmin=0.0, hmax=0.0, hstart=0.0, facmin=0.0, facmax=0.0, facrej=0.0,
                  facsafe=0.0) -> Tuple[List[int], List[float]]:
    """IPAR[20], RPAR[20] in the C layout; zero selects the reference default."""
    m = METHODS[method.lower()] if isinstance(method, str) else int(method)
    ipar = [0] * 20
    rpar = [0.0] * 20
    ipar[0] = 1 if autonomous else 0
    ipar[1] = 1 if scalar_tol else 0
    ipar[2] = int(max_steps)
    ipar[3] = m
    rpar[0:7] = [hmin, hmax, hstart, facmin, facmax, facrej, facsafe]
    return ipar, [float(x) for x in rpar]


def from_fortran(icntrl: Sequence[int], rcntrl: Sequence[float]) -> Tuple[List[int], List[float]]:
    """ICNTRL(1:20)/RCNTRL(1:20) (1-based in Fortran, given here as 0-based
    Python lists) to the C IPAR/RPAR layout."""
    ipar = [0] * 20
    rpar = [0.0] * 20
    ipar[0] = int(icntrl[0])
    ipar[1] = int(icntrl[1])
    ipar[2] = int(icntrl[3])
    ipar[3] = int(icntrl[2])
    for i in range(7):
        rpar[i] = float(rcntrl[i])
    return ipar, rpar
