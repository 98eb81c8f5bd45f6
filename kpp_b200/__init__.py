"""kpp_b200 -- batched Rosenbrock integration of KPP mechanisms on B200.

Components
  kpp_b200/gen/          kppcu, the KPP mechanism compiler (C++) that writes a
                         mechanism's rates, Fun, Jac_SP, sparse LU and solves as
                         sm_100a device code
  kpp_b200/csrc/         the hand-written CUDA Rosenbrock kernel and the C ABI
                         (include/kpp_b200.h)
  kpp_b200/mechanism.py  Python host layer over the C ABI (torch tensors)
  kpp_b200/controls.py   integrator controls (IPAR/RPAR, ICNTRL/RCNTRL)
  kpp_b200/build.py      build of kppcu and the per-mechanism libraries
"""
from .controls import IERR_TEXT, ISTATUS_NAMES, METHODS, from_fortran, make_controls
from .mechanism import KppError, Mechanism, RosenbrockResult, library_path, load

__all__ = ["Mechanism", "RosenbrockResult", "KppError", "load", "library_path",
           "make_controls", "from_fortran", "METHODS", "ISTATUS_NAMES", "IERR_TEXT"]
