"""KPP's own generator with kpp_b200's CUDA target (#LANGUAGE CUDA).

This is the generator route to the device code: KPP's generator, compiled
from its unchanged sources with the CUDA writer of kpp_b200/kppgen/code_cuda.c
added beside its C, Fortran and MATLAB writers, writes a mechanism's Fun,
Jac_SP, KppSolve and Update_RCONST as CUDA device templates (and pastes the
device util templates of kpp_b200/kppgen/util/, KppDecomp among them).  The
kppcu compiler (kpp_b200/gen/) is the default route; both emit the same
arithmetic (tests/test_kpp_route.py).  `python -m kpp_b200.build` builds, for
small_strato and saprc99 and whenever KPP's sources are found ($KPP_HOME, or
--kpp-home), a second library of each on this route,
libkpp_b200_<mech>_kpproute.so (--no-kpp-route skips it).

Steps, all under kpp_b200/_build/kppgen/ (git-ignored):
  1. src/      copy of $KPP_HOME/src with the four hooks that select the CUDA
               writer (hook() below: the CUDA_LANG value of `enum lang`,
               CmdLanguage's CUDA argument, the Use_CUDA prototype and the
               CUDA_LANG case of Generate()'s language switch);
  2. kpp       that copy compiled with code_cuda.c and the hand-written
               scanner/parser (frontend.c: flex, bison and libfl are absent);
  3. home/     a KPP home for the generator: models/ and examples/ of
               $KPP_HOME, util/ with the device templates (named as the
               generator looks them up), and empty int/none and drv/none
               (the kernel is the integrator);
  4. out/<mech>/  the generated files, with the host-side _Global.h and
               _Sparse.h replaced by empty headers (the device code reads no
               host globals) and route_includes.h, which includes the device
               files in order (kpp_b200/csrc/kpp_rosenbrock.cu includes it,
               then route_adapter.cuh).
"""
from __future__ import annotations

import hashlib
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
BUILD = PKG / "_build" / "kppgen"
GEN_SOURCES = ["code", "code_c", "code_f77", "code_f90", "code_matlab", "debug", "gen", "kpp",
               "scanner", "scanutil"]
UTIL = {"sutil": "sutil.cu", "blas": "blas.cu", "UserRateLaws": "UserRateLaws.cu",
        "UpdateSun": "UpdateSun.cu", "util": "util.cu"}


class RouteError(RuntimeError):
    pass


def _replace_once(text: str, old: str, new: str, where: str) -> str:
    if text.count(old) != 1:
        raise RouteError(f"{where}: expected one occurrence of {old!r}; the KPP sources differ "
                         f"from the version this hook was written for (KPP 3.5.0)")
    return text.replace(old, new, 1)


def hook(src: Path) -> None:
    """The four edits that let Generate() select the CUDA writer."""
    p = src / "gdata.h"
    p.write_text(_replace_once(p.read_text(), "MATLAB_LANG };", "MATLAB_LANG, CUDA_LANG };",
                               "gdata.h (enum lang)"))
    p = src / "code.h"
    p.write_text(_replace_once(p.read_text(), "void Use_MATLAB( char* rootFileName );",
                               "void Use_MATLAB( char* rootFileName );\n"
                               "void Use_CUDA( char* rootFileName );", "code.h"))
    p = src / "scanner.c"
    p.write_text(_replace_once(
        p.read_text(), '  ScanError("\'%s\': Unknown parameter for #LANGUAGE',
        '  if( EqNoCase( cmd, "CUDA" ) ) {\n    useLang = CUDA_LANG;\n    return;\n  }\n'
        '  ScanError("\'%s\': Unknown parameter for #LANGUAGE', "scanner.c (CmdLanguage)"))
    p = src / "gen.c"
    # the CUDA writer, then every generation decision as for C
    p.write_text(_replace_once(
        p.read_text(), "    case MATLAB_LANG: Use_MATLAB( rootFileName );\n                 break;",
        "    case MATLAB_LANG: Use_MATLAB( rootFileName );\n                 break;\n"
        "    case CUDA_LANG: Use_CUDA( rootFileName );\n"
        "                 useLang = C_LANG;\n                 break;", "gen.c (Generate)"))


def _digest(paths) -> str:
    h = hashlib.sha256()
    for p in sorted(str(x) for x in paths):
        h.update(p.encode())
        h.update(Path(p).read_bytes())
    return h.hexdigest()


def build_generator(kpp_home: str, force: bool = False) -> Path:
    """Compile KPP's generator with the CUDA target; returns the binary."""
    ksrc = Path(kpp_home) / "src"
    if not (ksrc / "gen.c").exists():
        raise RouteError(f"KPP sources not found under {ksrc}")
    inputs = [ksrc / f"{f}.c" for f in GEN_SOURCES] + list(ksrc.glob("*.h")) + [
        HERE / "code_cuda.c", HERE / "frontend.c", HERE / "y.tab.h", Path(__file__)]
    exe = BUILD / "kpp"
    stamp = BUILD / "kpp.stamp"
    key = _digest(inputs)
    if not force and exe.exists() and stamp.exists() and stamp.read_text() == key:
        return exe
    src = BUILD / "src"
    if src.exists():
        shutil.rmtree(src)
    src.mkdir(parents=True)
    for f in list(ksrc.glob("*.c")) + list(ksrc.glob("*.h")):
        shutil.copy(f, src / f.name)
    hook(src)
    cc = shutil.which("gcc") or "gcc"
    objs = []
    for name in GEN_SOURCES:
        o = BUILD / f"{name}.o"
        subprocess.run([cc, "-O", "-w", "-I", str(HERE), "-I", str(src), "-c", str(src / f"{name}.c"),
                        "-o", str(o)], check=True)
        objs.append(o)
    for path in (HERE / "code_cuda.c", HERE / "frontend.c"):
        o = BUILD / f"{path.stem}.o"
        subprocess.run([cc, "-O", "-Wall", "-Wno-unused-function", "-I", str(HERE), "-I", str(src),
                        "-c", str(path), "-o", str(o)], check=True)
        objs.append(o)
    subprocess.run([cc] + [str(o) for o in objs] + ["-lm", "-o", str(exe)], check=True)
    stamp.write_text(key)
    return exe


def make_home(kpp_home: str) -> Path:
    """A KPP home whose util/ holds the device templates."""
    home = BUILD / "home"
    if home.exists():
        shutil.rmtree(home)
    (home / "util").mkdir(parents=True)
    for sub in ("models", "examples"):
        if (Path(kpp_home) / sub).exists():
            os.symlink(Path(kpp_home).resolve() / sub, home / sub)
    for name, fname in UTIL.items():
        shutil.copy(HERE / "util" / fname, home / "util" / f"{name}.c")
    (home / "util" / "Makefile_c").write_text("# no Makefile for the CUDA target\n")
    for sub in ("int", "drv"):
        (home / sub).mkdir()
        (home / sub / "none.c").write_text("/* the kpp_b200 kernel integrates */\n")
    (home / "int" / "none.def").write_text("#INTFILE none\n")
    return home


def generate(mech: str, kpp_home: str, force: bool = False, hessian: bool = True) -> Path:
    """Run the generator with #LANGUAGE CUDA on one of KPP's models; returns
    the output directory (with route_includes.h).  hessian: #HESSIAN ON (the
    Hessian, Hess_Vec and HessTR_Vec of the discrete adjoint)."""
    exe = build_generator(kpp_home, force)
    home = make_home(kpp_home)
    out = BUILD / "out" / mech
    if out.exists():
        shutil.rmtree(out)
    out.mkdir(parents=True)
    model = f"#MODEL      {mech}\n"
    if mech == "mcm_isoprene":
        # KPP ships the MCM example for Fortran 90 only: the C translation the
        # kppcu route and the oracle read (kpp_b200/gen/mcm.py)
        from ..gen import mcm
        mcm.write(Path(kpp_home), out)
        model = "#INCLUDE    mcm_isoprene_c.eqn\n"
    (out / f"{mech}.kpp").write_text(
        f"#LANGUAGE   CUDA\n#DOUBLE     ON\n#INTEGRATOR none\n"
        f"#DRIVER     none\n#JACOBIAN   SPARSE_LU_ROW\n#HESSIAN    {'ON' if hessian else 'OFF'}\n"
        f"#STOICMAT   OFF\n"
        f"#MEX        OFF\n" + model)
    r = subprocess.run([str(exe), f"{mech}.kpp"], cwd=out, env={**os.environ, "KPP_HOME": str(home)},
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0 or not (out / f"{mech}_Function.cu").exists():
        raise RouteError(f"KPP's generator failed for {mech}:\n{r.stdout[-3000:]}")
    # the device code reads no host globals and has its own sparse tables
    for suffix in ("_Global.h", "_Sparse.h"):
        (out / f"{mech}{suffix}").write_text(
            f"/* {mech}{suffix}: host declarations, not part of the device code */\n")
    params = (out / f"{mech}_Parameters.h").read_text()
    macros = [m for m in re.findall(r"^#define\s+(\w+)\s", params, flags=re.M)
              if not m.startswith(("ind_", "indf_"))]
    lines = [f"// KPP's generator, #LANGUAGE CUDA, mechanism {mech}: its device files in order.",
             "// Generated by kpp_b200/kppgen/build.py.  Do not edit.", "#pragma once",
             f'#include "{mech}_Parameters.h"', f'#include "{mech}_JacobianSP.cu"',
             f'#include "{mech}_Function.cu"', f'#include "{mech}_Jacobian.cu"',
             f'#include "{mech}_LinearAlgebra.cu"', f'#include "{mech}_Rates.cu"']
    nhess = re.search(r"^#define\s+NHESS\s+(\d+)", params, flags=re.M)
    if hessian and nhess:
        lines += [f'#include "{mech}_HessianSP.cu"', f'#include "{mech}_Hessian.cu"',
                  f"#define KPP_NHESS {nhess.group(1)}  // entries of the sparse Hessian"]
    lines += ["// the sizes are kpp_b200's own constants from here on"]
    lines += [f"#undef {m}" for m in macros]
    (out / "route_includes.h").write_text("\n".join(lines) + "\n")
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("mechs", nargs="+")
    ap.add_argument("--kpp-home", default=os.environ.get("KPP_HOME", ""))
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    for m in a.mechs:
        print(generate(m, a.kpp_home, a.force))


if __name__ == "__main__":
    sys.exit(main())
