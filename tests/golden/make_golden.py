"""Write the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own KPP-generated C code built by oracle/build_ref.sh
(oracle/_ref/<mech>/libkppref_<mech>.so, the reference Rosenbrock of
int/rosenbrock.c driven by oracle/refkpp/batch_driver.c) on small seeded
batches and stores inputs and outputs:

  structure_<mech>.json   species order, sizes and the sparse LU pattern of
                          the reference generator's output
  funjac_<mech>.npz       rate constants, Fun and Jac_SP of a few cells
  integrate_<mech>.npz    chained chemistry steps of a small batch: inputs,
                          VAR after every step, ISTATUS, RSTATUS and IERR, and
                          var_alt [step, 5, NVAR, cells]: the same steps by the
                          reference under other valid last-ulp roundings
                          (oracle_lib.alternates)

Usage (needs the oracle build, i.e. the reference sources at build time):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parents[1]))

from oracle_lib import OracleLib, alternates, ensure_built  # noqa: E402
from kpp_b200 import workloads  # noqa: E402


class _MechView:
    """The parts of a mechanism the workload generator needs, from the oracle."""

    def __init__(self, o: OracleLib):
        self.o = o
        self.nvar = o.nvar
        self.species = o.species

    def initial_values(self):
        c, cf = self.o.initial_values()
        return list(c), cf


def structure(o: OracleLib) -> dict:
    irow, icol, crow, diag = o.lu_pattern()
    return {"mechanism": o.mech, "nvar": o.nvar, "nfix": o.nfix, "nspec": o.nspec,
            "nreact": o.nreact, "lu_nonzero": o.lu_nonzero, "species": o.species,
            "lu_irow": irow.tolist(), "lu_icol": icol.tolist(), "lu_crow": crow.tolist(),
            "lu_diag": diag.tolist()}


def funjac(o: OracleLib, wl: workloads.Workload, ncells: int, times) -> dict:
    out = {"var": wl.var[:, :ncells], "fix": wl.fix[:, :ncells], "temp": wl.temp[:ncells],
           "cfactor": (wl.cfactor[:ncells] if wl.cfactor is not None else np.full(ncells, o.initial_values()[1])),
           "sun": (wl.sun[:ncells] if wl.sun is not None else np.full(ncells, -1.0)),
           "time": np.asarray(times[:ncells], dtype=np.float64)}
    rc, vd, jv = [], [], []
    for c in range(ncells):
        r, v, j = o.fun_jac(out["var"][:, c], out["fix"][:, c], out["temp"][c], out["cfactor"][c],
                            None if out["sun"][c] < 0 else out["sun"][c], out["time"][c])
        rc.append(r); vd.append(v); jv.append(j)
    out["rconst"] = np.stack(rc, 1)
    out["vdot"] = np.stack(vd, 1)
    out["jvs"] = np.stack(jv, 1)
    return out


def integrate_chain(o: OracleLib, wl: workloads.Workload, nsteps: int) -> dict:
    var = wl.var.copy()
    hstart = np.zeros(wl.ncells)
    res = {"var0": wl.var, "fix": wl.fix, "temp": wl.temp,
           "cfactor": wl.cfactor if wl.cfactor is not None else np.zeros(0),
           "sun": wl.sun if wl.sun is not None else np.zeros(0),
           "tstart": wl.tstart, "dt": np.array(wl.dt), "atol": wl.atol, "rtol": wl.rtol,
           "ipar": np.array(wl.ipar, np.int32), "rpar": np.array(wl.rpar)}
    vs, ists, rsts, ierrs, alts = [], [], [], [], []
    for k in range(nsteps):
        t0, t1 = wl.step_bounds(k)
        prev = var.copy()
        var, ist, rst, ierr = o.integrate(var, wl.fix, wl.temp, t0, t1, wl.atol, wl.rtol,
                                          wl.ipar, wl.rpar, cfactor=wl.cfactor, sun=wl.sun,
                                          hstart=hstart, which="ref")
        # the same step by the reference under other valid last-ulp roundings
        # (FMA contraction; SUN one ulp up / down; the
        # step controller's pow() one ulp up / down), which measures how far the
        # result itself moves under last-ulp perturbations
        va = alternates(o.mech, prev, wl.fix, wl.temp, t0, t1, wl.atol, wl.rtol, wl.ipar,
                        wl.rpar, cfactor=wl.cfactor, sun=wl.sun, hstart=hstart)
        hstart = rst[1].copy()
        vs.append(var.copy()); ists.append(ist); rsts.append(rst); ierrs.append(ierr)
        alts.append(va)
    res["var"] = np.stack(vs)
    res["var_alt"] = np.stack(alts)
    res["istatus"] = np.stack(ists)
    res["rstatus"] = np.stack(rsts)
    res["ierr"] = np.stack(ierrs)
    return res


def main():
    if not ensure_built():
        raise SystemExit("oracle libraries are not built (reference sources needed)")
    # small_strato: 64 cells, 6 chained chemistry steps of 1200 s
    o = OracleLib("small_strato")
    (HERE / "structure_small_strato.json").write_text(json.dumps(structure(o), indent=1))
    wl = workloads.for_mechanism(_MechView(o), "small_strato", 64)
    np.savez_compressed(HERE / "funjac_small_strato.npz",
                        **funjac(o, wl, 16, wl.tstart + 1000.0))
    np.savez_compressed(HERE / "integrate_small_strato.npz",
                        **integrate_chain(o, wl, 6))
    # saprc99: 24 cells, 2 chained steps of 600 s, SZA uniform in 0-95 degrees
    o = OracleLib("saprc99")
    (HERE / "structure_saprc99.json").write_text(json.dumps(structure(o), indent=1))
    wl = workloads.for_mechanism(_MechView(o), "saprc99", 24)
    np.savez_compressed(HERE / "funjac_saprc99.npz", **funjac(o, wl, 6, wl.tstart))
    np.savez_compressed(HERE / "integrate_saprc99.npz",
                        **integrate_chain(o, wl, 2))
    # MCM isoprene (translated from examples/mcm): 8 cells, 2 chained
    # Rodas4 steps of 300 s
    o = OracleLib("mcm_isoprene")
    st = structure(o)
    st["nfix"] = o.nspec - o.nvar  # KPP's C model pads NFIX to 1 when it is 0
    (HERE / "structure_mcm_isoprene.json").write_text(json.dumps(st, indent=1))
    wl = workloads.for_mechanism(_MechView(o), "mcm_isoprene", 8)
    np.savez_compressed(HERE / "funjac_mcm_isoprene.npz", **funjac(o, wl, 3, wl.tstart))
    np.savez_compressed(HERE / "integrate_mcm_isoprene.npz", **integrate_chain(o, wl, 2))
    for p in sorted(HERE.glob("*.*")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
