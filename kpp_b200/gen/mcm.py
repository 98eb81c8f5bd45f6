"""MCM isoprene (KPP's examples/mcm) as a C / CUDA-language KPP mechanism.

KPP ships the Master Chemical Mechanism example for the Fortran 90 target
only: its rate constants are Fortran expressions over named constants
(KRO2NO, KMT01, ...) and photolysis frequencies J(...) that the module
constants_mcm.f90 computes from TEMP, M and the solar zenith angle, plus an
RO2 sum over the peroxy radicals in an `#INLINE F90_RCONST` block; the
example driver (driver_mcm.f90) sets M, O2, N2 and H2O.  This module writes,
from those files, the same species and equations with every rate translated
to C (kpp_b200/gen/fortran.py, Fortran literal kinds and precedence kept)
and inline rate prologues (`mcm_isoprene_cuda.eqn` for kppcu: split into
CUDA_RCONST_STATIC / _SUN / CUDA_RCONST by dependence, so that kppcu hoists
the rates that do not read the concentrations; `mcm_isoprene_c.eqn` for the
reference generator: one C_RCONST block) that compute, per cell, what the
Fortran module and driver compute:

  M = CFACTOR (molec/cm3, per cell); O2, N2, H2O from M as the driver does;
  cos(zenith) = SUN (per cell; the J formulas only use cos(zenith));
  every statement of define_constants_mcm, in order;
  RO2 = the inline block's sum of concentrations (the accepted state C, the
  array Update_RCONST reads in the reference).

The reference generator reads the file for the oracle (`#LANGUAGE C`), kppcu
for the device code (`#LANGUAGE CUDA`).  Nothing of the mechanism is stored
in this repository: the file is produced at build time from KPP_HOME.

  python -m kpp_b200.gen.mcm --home KPP_HOME --out DIR
"""
from __future__ import annotations

import argparse
import re
from pathlib import Path

from .fortran import F64, Context, FortranError, join_continuations, translate_assignment
from .fortran import translate_expr

EXAMPLE = Path("examples") / "mcm"
DRIVER_ENV = ("O2", "N2", "H2O")  # derived from M in the example driver


def _j_params(src: str) -> dict:
    out = {}
    for m in re.finditer(r"INTEGER\s*,\s*PARAMETER\s*::\s*(J_\w+)\s*=\s*(\d+)", src, re.I):
        out[m.group(1).upper()] = int(m.group(2))
    return out


def _constants_body(src: str) -> list:
    m = re.search(r"SUBROUTINE\s+define_constants_mcm\s*\(\s*\)(.*?)END\s+SUBROUTINE", src,
                  re.S | re.I)
    if not m:
        raise FortranError("define_constants_mcm not found")
    return join_continuations(m.group(1).splitlines())


def _driver_env(src: str) -> list:
    stmts = []
    for line in join_continuations(src.splitlines()):
        m = re.match(r"^(\w+)\s*=\s*(.+)$", line)
        if m and m.group(1).upper() in DRIVER_ENV and re.search(r"\bM\b", m.group(2)):
            stmts.append(line)
    if len(stmts) != len(DRIVER_ENV):
        raise FortranError("driver: expected O2, N2 and H2O as multiples of M")
    return stmts


def _inline_blocks(eqn: str):
    """(text without the F90 inline blocks, RO2 statements of F90_RCONST)."""
    ro2 = []
    pat = re.compile(r"#INLINE\s+(F90_\w+)(.*?)#ENDINLINE[^\n]*\n", re.S)
    for m in pat.finditer(eqn):
        if m.group(1) == "F90_RCONST":
            for st in join_continuations(m.group(2).splitlines()):
                if st.upper().startswith("CALL "):
                    continue
                ro2.append(st)
    return pat.sub("", eqn), ro2


def rconst_parts(constants_src: str, driver_src: str, ro2_stmts: list, lang: str):
    """The per-cell rate-constant prologue in C, split by what it depends on:
    (TEMP / CFACTOR only: M, O2, N2, H2O and the named constants; SUN: the
    photolysis frequencies J; the concentrations: RO2).  `lang` 'C' reads the
    reference's global C array, 'CUDA' the VAR accessor of the device rate
    functions."""
    jp = _j_params(constants_src)
    nj = max(jp.values()) + 1 if jp else 1
    conc = "C" if lang == "C" else "VAR"
    ctx = Context(arrays={"J": lambda n, i: f"J[{i.text}]",
                          "C": lambda n, i: f"{conc}[{i.text}]"},
                  int_params=jp)
    static = ["  /* MCM rate-constant environment of the cell, translated from",
              "     examples/mcm/constants_mcm.f90 and driver_mcm.f90 */",
              "  double M = CFACTOR;"]
    for st in _driver_env(driver_src):
        c, name = translate_assignment(st, ctx)
        static.append(f"  double {c}")
    names, kbody, jbody = [], [], []
    for st in _constants_body(constants_src):
        st = re.sub(r"cos\s*\(\s*zenith\s*\)", "SUN", st, flags=re.I)
        if re.search(r"\bzenith\b", st, re.I):
            raise FortranError(f"zenith used other than as cos(zenith): {st}")
        c, name = translate_assignment(st, ctx)
        if name.upper() == "J":
            jbody.append("  " + c)
            continue
        if re.search(r"\bSUN\b|\bJ\s*\(", st):
            raise FortranError(f"a named constant depends on the sun: {st}")
        if name not in names:
            names.append(name)
        kbody.append("  " + c)
    for k in range(0, len(names), 8):
        static.append("  double " + ", ".join(names[k:k + 8]) + ";")
    static += kbody
    static.append("  (void)M;" + "".join(f" (void){n};" for n in DRIVER_ENV))
    sun = [f"  double J[{nj}];"] + jbody + ["  (void)J;"]
    dyn = []
    for st in ro2_stmts:
        dyn += _sum_lines(st, conc)
    dyn.append("  (void)RO2;")
    return ("\n".join(static) + "\n", "\n".join(sun) + "\n", "\n".join(dyn) + "\n")


def _sum_lines(stmt: str, conc: str, per_line: int = 6) -> list:
    """`RO2 = C(ind_a) + C(ind_b) + ...` as C lines of at most a few terms
    (the reference generator keeps 1000 characters of an inline line), adding
    left to right exactly as the single Fortran expression does."""
    m = re.match(r"^(\w+)\s*=\s*(.+)$", stmt)
    terms = [t.strip() for t in m.group(2).split("+")]
    idx = []
    for t in terms:
        mt = re.fullmatch(r"C\(\s*(ind_\w+)\s*\)", t, re.I)
        if not mt:
            raise FortranError(f"{m.group(1)}: expected a sum of C(ind_*) terms, got {t!r}")
        idx.append(mt.group(1))
    name = m.group(1)
    refs = [f"{conc}[{i}]" for i in idx]
    out = [f"  double {name} = {refs[0]};"]
    for k in range(1, len(refs), per_line):
        out.append(f"  {name} = " + "(" * len(refs[k:k + per_line]) + name
                   + "".join(f" + {r})" for r in refs[k:k + per_line]) + ";")
    return out


def translate_equations(text: str):
    """Every `<tag> reactants = products : rate ;` line with its rate in C.
    Returns (text with the translated rates, text with every rate replaced by
    MCMR[k], the translated rates in equation order)."""
    ctx = Context(arrays={"J": lambda n, i: f"J[{i.text}]"}, int_params={})
    full, ref, rates, in_eqn = [], [], [], False
    for line in text.splitlines(keepends=True):
        s = line.strip()
        if s.upper().startswith("#EQUATIONS"):
            in_eqn = True
            full.append(line)
            ref.append(line)
            continue
        if in_eqn and s.startswith("#"):
            in_eqn = False
        if in_eqn and ":" in line and ";" in line:
            head, rest = line.split(":", 1)
            rate, tail = rest.rsplit(";", 1)
            e = translate_expr(rate.strip(), ctx)
            full.append(f"{head}: ({e.text}) ;{tail}")
            ref.append(f"{head}: MCMR[{len(rates)}] ;{tail}")
            rates.append(e.text)
            continue
        full.append(line)
        ref.append(line)
    return "".join(full), "".join(ref), rates


def write(home: Path, out_dir: Path) -> Path:
    """Writes mcm_isoprene_cuda.eqn (rates as C expressions, for kppcu) and
    mcm_isoprene_c.eqn (for the reference generator, whose C writer breaks
    long assignments at operators it encodes itself and so would cut a
    translated expression inside a token: there every rate is MCMR[k],
    computed by the same expression in the C_RCONST block)."""
    ex = Path(home) / EXAMPLE
    eqn = (ex / "mcm_isoprene.eqn").read_text(encoding="utf-8", errors="replace")
    constants = (ex / "constants_mcm.f90").read_text()
    driver = (ex / "driver_mcm.f90").read_text()
    # J(J_NAME) in rates: resolve the names to their integer parameters first
    jp = _j_params(constants)
    eqn = re.sub(r"J\(\s*(J_\w+)\s*\)", lambda m: f"J({jp[m.group(1).upper()]})", eqn)
    body, ro2 = _inline_blocks(eqn)
    full, ref, rates = translate_equations(body)
    head = ("{ Generated by kpp_b200/gen/mcm.py from KPP's examples/mcm (Fortran 90 rates\n"
            "  translated to C); do not edit. }\n")
    out_dir.mkdir(parents=True, exist_ok=True)
    for name, text, lang in (("mcm_isoprene_cuda.eqn", full, "CUDA"),
                             ("mcm_isoprene_c.eqn", ref, "C")):
        st, sn, dy = rconst_parts(constants, driver, ro2, lang)
        if lang == "C":
            # the reference evaluates everything in Update_RCONST, in order
            blocks = (f"#INLINE C_RCONST\n{st}{sn}{dy}  double MCMR[{len(rates)}];\n"
                      + "".join(f"  MCMR[{k}] = {r};\n" for k, r in enumerate(rates))
                      + "#ENDINLINE\n")
        else:
            # kppcu hoists rates by class: a rate using only the static names
            # is computed once per cell, one using J once per SUN value
            blocks = (f"#INLINE CUDA_RCONST_STATIC\n{st}#ENDINLINE\n"
                      f"#INLINE CUDA_RCONST_SUN\n{sn}#ENDINLINE\n"
                      f"#INLINE CUDA_RCONST\n{dy}#ENDINLINE\n")
        i = text.upper().index("#EQUATIONS")
        (out_dir / name).write_text(head + text[:i] + blocks + text[i:])
    return out_dir / "mcm_isoprene_cuda.eqn"


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--home", required=True)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    print(write(Path(a.home), Path(a.out)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
