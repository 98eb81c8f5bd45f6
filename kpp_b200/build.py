"""Build the native parts of kpp_b200.

  1. kppcu, the KPP mechanism compiler (C++, kpp_b200/gen/), with g++.
  2. For each mechanism in kpp_b200/mechanisms/: kppcu writes the mechanism's
     CUDA device code (kpp_b200/_gen/<mech>.cuh), and nvcc builds the batched
     Rosenbrock library kpp_b200/lib/libkpp_b200_<mech>.so for sm_100a.
  3. For the mechanisms of KPP_ROUTE, when KPP's sources are at hand: KPP's
     own generator with kpp_b200's CUDA target (kpp_b200/kppgen) writes the
     arithmetic, and the same kernels are built on it into
     libkpp_b200_<mech>_kpproute.so.

The kernel source is compiled once per part (the C ABI, and one part per
Rosenbrock method) in parallel, then linked.  Builds are incremental: a
stamp holding a hash of every input and flag skips up-to-date libraries.

Mechanism sources (.def/.spc/.eqn) are looked up in the directory of the
mechanism file and under $KPP_HOME/models (KPP's own layout).  Without them
(for example on a machine that received prebuilt libraries) the existing
libraries are kept; a missing library is an error.

Usage: python -m kpp_b200.build [mech ...] [--all] [--force] [--jobs N] [--kpp-home DIR]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import json
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
GEN_SRC = PKG / "gen"
CSRC = PKG / "csrc"
MECH_DIR = PKG / "mechanisms"
BUILD = PKG / "_build"
GEN_OUT = PKG / "_gen"
LIB = PKG / "lib"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no FMA contraction, so the double arithmetic rounds like the
# reference C code built without FMA (x86-64 gcc -O).
# -fvisibility=hidden: only the C ABI (declared with default visibility in
# include/kpp_b200.h) is exported, so the function-local statics of the
# launchers (per-device set-up) are not merged across mechanism libraries
# loaded in one process.
NVCC_FLAGS = ["-O3", "--fmad=false", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-diag-suppress", "177"]
METHOD_PARTS = [1, 2, 3, 4, 5]
SDIRK_PART = 6  # the SDIRK integrator
RK_PART = 7     # the Runge-Kutta integrator (complex LU from <mech>_cmplx.cuh)
ADJ_PART = 8    # the Rosenbrock discrete adjoint (generator route with the Hessian only)
# Mechanisms at or above this LU size keep per-cell work arrays in the
# cell-fastest global scratch layout instead of thread-local arrays.
SCRATCH_LU_NONZERO = 200


_LINE_MARKER = re.compile(rb"\s*#\s*(line\b|\d)")

def default_kpp_home() -> str:
    """KPP's source tree (models/, examples/) from $KPP_HOME; empty when unset,
    and the build then keeps the prebuilt libraries."""
    return os.environ.get("KPP_HOME", "")


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return path


def _hash_files(paths, extra: str = "") -> str:
    h = hashlib.sha256(extra.encode())
    for p in sorted(str(x) for x in paths):
        h.update(p.encode())
        h.update(Path(p).read_bytes())
    return h.hexdigest()


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(map(str, cmd))}\n{r.stdout}")
    return r.stdout


def build_kppcu(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    exe = BUILD / "kppcu"
    srcs = sorted(GEN_SRC.glob("*.cpp")) + sorted(GEN_SRC.glob("*.hpp"))
    stamp = BUILD / "kppcu.stamp"
    digest = _hash_files(srcs)
    if not force and exe.exists() and stamp.exists() and stamp.read_text() == digest:
        return exe
    cxx = shutil.which("g++") or "g++"
    _run([cxx, "-std=c++17", "-O2", "-Wall", "-Wextra", "-o", str(exe)]
         + [str(p) for p in GEN_SRC.glob("*.cpp")])
    stamp.write_text(digest)
    return exe


# Mechanisms KPP ships for another target language only: their sources are
# translated to a C-language KPP mechanism first (kpp_b200/gen/mcm.py).
TRANSLATED = {"mcm_isoprene": ("examples/mcm", ("mcm_isoprene.eqn", "constants_mcm.f90",
                                                "driver_mcm.f90"))}


def mechanism_sources(mech: str, kpp_home: str):
    """Files kppcu reads for a mechanism (for the incremental-build hash)."""
    files = [MECH_DIR / f"{mech}.kpp"]
    if mech in TRANSLATED:
        sub, names = TRANSLATED[mech]
        ex = Path(kpp_home) / sub if kpp_home else None
        if ex and all((ex / n).exists() for n in names):
            files += [ex / n for n in names] + [GEN_SRC / "fortran.py", GEN_SRC / "mcm.py"]
            atoms = Path(kpp_home) / "models" / "atoms"
            if atoms.exists():
                files.append(atoms)
        return files
    if kpp_home:
        for ext in (".def", ".spc", ".eqn"):
            p = Path(kpp_home) / "models" / f"{mech}{ext}"
            if p.exists():
                files.append(p)
        inc = Path(kpp_home) / "models" / "atoms.kpp"
        if inc.exists():
            files.append(inc)
    return files


def generate(mech: str, kpp_home: str, force: bool = False) -> Path | None:
    """Run kppcu; returns the generated header, or None without sources."""
    src = mechanism_sources(mech, kpp_home)
    if len(src) < 2:
        return None
    GEN_OUT.mkdir(exist_ok=True)
    exe = build_kppcu(force)
    out = GEN_OUT / mech
    stamp = GEN_OUT / f"{mech}.stamp"
    digest = _hash_files(src + [exe])
    if not force and stamp.exists() and stamp.read_text() == digest and (GEN_OUT / f"{mech}.cuh").exists():
        return GEN_OUT / f"{mech}.cuh"
    top = MECH_DIR / f"{mech}.kpp"
    if mech in TRANSLATED:
        from .gen import mcm
        src_dir = GEN_OUT / f"{mech}_src"
        mcm.write(Path(kpp_home), src_dir)
        shutil.copy(top, src_dir / top.name)
        top = src_dir / top.name
    _run([str(exe), str(top), "-o", str(out), "--home", kpp_home, "--root", mech])
    stamp.write_text(digest)
    return GEN_OUT / f"{mech}.cuh"


def library_path(mech: str, route: str = "kppcu") -> Path:
    """The mechanism library; route "kpp": built on the arithmetic that KPP's
    own generator writes with #LANGUAGE CUDA (kpp_b200/kppgen)."""
    return LIB / (f"libkpp_b200_{mech}.so" if route == "kppcu" else f"libkpp_b200_{mech}_kpproute.so")


def compile_library(mech: str, header: Path, jobs: int, force: bool = False,
                    route_dir: Path | None = None) -> Path:
    """nvcc each part (the C ABI, one part per Rosenbrock method, the SDIRK
    and the Runge-Kutta integrators) in parallel and link the shared library.  A part is recompiled only when its own
    preprocessed source or flags change (large mechanisms take many minutes
    per part), so a change confined to the C ABI rebuilds part 0 alone."""
    LIB.mkdir(exist_ok=True)
    objdir = BUILD / (mech if route_dir is None else f"{mech}_kpproute")
    objdir.mkdir(parents=True, exist_ok=True)
    meta = json.loads((GEN_OUT / f"{mech}.json").read_text())
    defines = [f'-DKPP_MECH_HEADER="{header}"']
    if meta["lu_nonzero"] >= SCRATCH_LU_NONZERO:
        defines.append("-DKPP_SCRATCH")
    if route_dir is not None:
        defines += ["-DKPP_EXTERNAL_ARITHMETIC",
                    f'-DKPP_ROUTE_INCLUDE="{route_dir / "route_includes.h"}"',
                    "-I", str(route_dir), "-I", str(PKG / "kppgen"), "-I", str(CSRC)]
    host_header = GEN_OUT / f"{mech}_host.h"
    lib = library_path(mech, "kppcu" if route_dir is None else "kpp")
    parts = [0] + METHOD_PARTS + [SDIRK_PART, RK_PART]
    if route_dir is not None and "KPP_NHESS" in (route_dir / "route_includes.h").read_text():
        parts.append(ADJ_PART)

    def part_flags(part: int):
        f = ARCH + NVCC_FLAGS + defines + [f"-DKPP_PART={part}", "-I", str(GEN_OUT)]
        if part == 0 and host_header.exists():
            f.append(f'-DKPP_HOST_HEADER="{host_header}"')
        if part == 0:
            f.append(f'-DKPP_ADJ_HEADER="{header.with_name(header.stem + "_adj.cuh")}"')
        if part == RK_PART:
            f.append(f'-DKPP_CMPLX_HEADER="{header.with_name(header.stem + "_cmplx.cuh")}"')
        return f

    def compile_part(part: int):
        obj = objdir / f"part{part}.o"
        flags = part_flags(part)
        pre = subprocess.run([nvcc(), "-E"] + flags + [str(CSRC / "kpp_rosenbrock.cu")],
                             capture_output=True, check=True).stdout
        # the code only: line markers (`# 12 "file"`, `#line`) and blank lines
        # do not change what is compiled (comments are already gone); pragmas
        # do and are kept
        code = b"\n".join(ln for ln in pre.splitlines()
                           if ln.strip() and not _LINE_MARKER.match(ln))
        digest = hashlib.sha256(code + " ".join(flags).encode()).hexdigest()
        stamp = objdir / f"part{part}.stamp"
        if not force and obj.exists() and stamp.exists() and stamp.read_text() == digest:
            return obj, False
        _run([nvcc()] + flags + ["-c", str(CSRC / "kpp_rosenbrock.cu"), "-o", str(obj)])
        stamp.write_text(digest)
        return obj, True

    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        results = list(ex.map(compile_part, parts))
    if any(rebuilt for _, rebuilt in results) or not lib.exists():
        _run([nvcc()] + ARCH + ["-shared", "-o", str(lib)] + [str(o) for o, _ in results]
             + ["-lcudart"])
    params = GEN_OUT / f"{mech}_Parameters.h"
    if params.exists():
        shutil.copy(params, LIB / f"kpp_b200_{mech}_Parameters.h")
    return lib


def build_util(force: bool = False) -> Path:
    """libkpp_b200_util.so: measurement helpers (FP64 peak)."""
    LIB.mkdir(exist_ok=True)
    BUILD.mkdir(exist_ok=True)
    src = CSRC / "kpp_util.cu"
    lib = LIB / "libkpp_b200_util.so"
    flags = ARCH + ["-O3", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                    "-lineinfo"]
    stamp = BUILD / "util.stamp"
    digest = _hash_files([src, CSRC / "kpp_ratelaws.cuh"], " ".join(flags))
    if not force and lib.exists() and stamp.exists() and stamp.read_text() == digest:
        return lib
    _run([nvcc()] + flags + [str(src), "-o", str(lib)])
    stamp.write_text(digest)
    return lib


def build_sched(force: bool = False) -> Path:
    """libkpp_b200_sched.so: the learned scheduler (features, BF16 tensor-core
    MLP, training kernels, scheduling pass); mechanism independent."""
    LIB.mkdir(exist_ok=True)
    BUILD.mkdir(exist_ok=True)
    src = CSRC / "kpp_sched.cu"
    deps = [src, CSRC / "kpp_ratelaws.cuh", INCLUDE / "kpp_sched.h"]
    lib = LIB / "libkpp_b200_sched.so"
    flags = ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-lineinfo",
                    "-I", str(INCLUDE), "-I", str(CSRC)]
    stamp = BUILD / "sched.stamp"
    digest = _hash_files(deps, " ".join(flags))
    if not force and lib.exists() and stamp.exists() and stamp.read_text() == digest:
        return lib
    _run([nvcc()] + flags + [str(src), "-o", str(lib)])
    stamp.write_text(digest)
    return lib


# Mechanisms whose library is also built on the KPP generator route (the
# arithmetic written by KPP's own generator with #LANGUAGE CUDA), when KPP's
# sources are at hand.
KPP_ROUTE = ("small_strato", "saprc99")


# Mechanisms built only when named (`python -m kpp_b200.build <mech>` or
# `--all`), or once their library exists.  None at present: MCM isoprene's LU
# and solve are loops over the LU tables (kppcu), so it builds with the rest.
ON_REQUEST: set = set()


def all_mechanisms():
    return sorted(p.stem for p in MECH_DIR.glob("*.kpp"))


def default_mechanisms():
    return [m for m in all_mechanisms() if m not in ON_REQUEST or library_path(m).exists()]


def build(mechs=None, force: bool = False, jobs: int | None = None, verbose: bool = True,
          kpp_home: str | None = None, route: bool = True):
    kpp_home = kpp_home if kpp_home is not None else default_kpp_home()
    jobs = jobs or os.cpu_count() or 4
    mechs = mechs or default_mechanisms()
    built = {"util": build_util(force), "sched": build_sched(force)}
    for mech in mechs:
        header = generate(mech, kpp_home, force)
        if header is None:
            lib = library_path(mech)
            if not lib.exists():
                raise RuntimeError(f"no mechanism sources for {mech} (KPP_HOME={kpp_home!r}) "
                                   f"and no prebuilt {lib}")
            built[mech] = lib
            continue
        built[mech] = compile_library(mech, header, jobs, force)
        if verbose:
            print(f"kpp_b200.build: {mech} -> {built[mech]}", flush=True)
        if mech in KPP_ROUTE and route:
            from .kppgen import build as kppgen
            out = kppgen.generate(mech, kpp_home, force)
            built[f"{mech}_kpproute"] = compile_library(mech, header, jobs, force, route_dir=out)
            if verbose:
                print(f"kpp_b200.build: {mech} (KPP generator route) -> "
                      f"{built[f'{mech}_kpproute']}", flush=True)
    return built


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("mechs", nargs="*")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--all", action="store_true", help="also the on-request mechanisms")
    ap.add_argument("--kpp-home", default=None,
                    help="KPP source tree with models/ and examples/ (default: $KPP_HOME)")
    ap.add_argument("--no-kpp-route", dest="route", action="store_false",
                    help="skip the libraries built on KPP's own generator (#LANGUAGE CUDA)")
    a = ap.parse_args(argv)
    build(a.mechs or (all_mechanisms() if a.all else None), force=a.force, jobs=a.jobs,
          kpp_home=a.kpp_home, route=a.route)


if __name__ == "__main__":
    sys.exit(main())
