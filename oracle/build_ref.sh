#!/usr/bin/env bash
# Build the oracle: the reference KPP generator and, for each mechanism, the
# reference's own KPP-generated C model with the reference Rosenbrock
# integrator, plus the CPU restatement (oracle/ros_oracle.c).
#
# ORACLE INFRASTRUCTURE ONLY.  Outputs go to oracle/_ref/ (git-ignored; the
# built files travel with the repository snapshot to the GPU machine, where
# the reference sources are absent and only these prebuilt libraries are used).
#
#   oracle/_ref/kpp                               reference generator
#   oracle/_ref/<mech>/<mech>_*.c|h               reference-generated model
#   oracle/_ref/<mech>/libkppref_<mech>.so        -O (reference flags, util/Makefile_c:3)
#   oracle/_ref/<mech>/libkppref_<mech>_O3.so     -O3 -march=x86-64-v3 (FMA contraction:
#                                                 the same code with another valid rounding)
#   oracle/_ref/<mech>/libkppref_<mech>_cs.so     Update_SUN's cos() one ulp on request
#   oracle/_ref/<mech>_sdirk/libkppsd_<mech>[_O3|_pw].so  the model with the reference
#                                                 SDIRK integrator (int/sdirk.c)
#   oracle/_ref/<mech>_rk/libkpprk_<mech>[_O3|_pw].so  ... with the reference Runge-Kutta
#                                                 integrator (int/runge_kutta.c)
#   oracle/_ref/<mech>_adj/libkppadj_<mech>[_O3|_pw].so  ... with the reference Rosenbrock
#                                                 adjoint (int/rosenbrock_adj.c) and Hessian
#
# The generator is compiled from the unchanged sources in $KPP_REF/src; only
# the flex/bison front end is replaced by kpp_b200/kppgen/frontend.c because
# flex, bison and libfl are not installed.  Usage:
#   oracle/build_ref.sh [KPP_REF=/path/to/reference] [mech ...]
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
FRONT="$HERE/../kpp_b200/kppgen"  # the hand-written scanner/parser of the KPP language
KPP_REF="${KPP_REF:-/root/reference}"
OUT="$HERE/_ref"
MECHS=("$@")
if [ ${#MECHS[@]} -eq 0 ]; then MECHS=(small_strato saprc99 mcm_isoprene); fi

if [ ! -d "$KPP_REF/src" ]; then
  echo "build_ref: reference sources not found at $KPP_REF; keeping prebuilt $OUT" >&2
  exit 0
fi

CC="${CC:-gcc}"
mkdir -p "$OUT/obj"
# the source tree the tests read the reference's mechanisms from
echo "$KPP_REF" > "$OUT/kpp_home"

# ---- 1. the generator -------------------------------------------------------
GEN_SRCS=(code code_c code_f77 code_f90 code_matlab debug gen kpp scanner scanutil)
for f in "${GEN_SRCS[@]}"; do
  "$CC" -O -w -I"$FRONT" -I"$KPP_REF/src" -c "$KPP_REF/src/$f.c" -o "$OUT/obj/$f.o"
done
"$CC" -O -Wall -Wno-unused-function -I"$FRONT" -I"$KPP_REF/src" \
  -c "$FRONT/frontend.c" -o "$OUT/obj/frontend.o"
"$CC" "$OUT"/obj/*.o -lm -o "$OUT/kpp"

# ---- 2. per-mechanism reference model ---------------------------------------
# build_integrator_model MECH INTEGRATOR DRIVER TAG PREFIX [HESSIAN]: the model with
# another reference integrator and its batch driver (refkpp/DRIVER.c) in
# oracle/_ref/MECH_TAG/: libPREFIX_MECH.so (reference flags), _O3 (FMA
# contraction) and _pw (the integrator's pow() through the driver's
# kppref_pow, refkpp/pow_knob.h, and Update_SUN's cos() through kppref_cos,
# refkpp/cos_knob.h; each can move its result one ulp: other valid
# roundings of pow and cos).
build_integrator_model() {
  local mech="$1" integ="$2" driver="$3" tag="$4" prefix="$5" hessian="${6:-OFF}"
  local ds="$OUT/${mech}_${tag}"
  local model="#MODEL      $mech"
  rm -rf "$ds"
  mkdir -p "$ds"
  if [ "$mech" = "mcm_isoprene" ]; then
    # the translated MCM (kpp_b200/gen/mcm.py), included after the SUN override
    (cd "$HERE/.." && python -m kpp_b200.gen.mcm --home "$KPP_REF" --out "$ds" > /dev/null)
    model=""
  fi
  cat > "$ds/$mech.kpp" <<EOF
$model
#LANGUAGE   C
#DOUBLE     ON
#INTEGRATOR $integ
#DRIVER     $HERE/refkpp/$driver
#JACOBIAN   SPARSE_LU_ROW
#HESSIAN    $hessian
#STOICMAT   OFF
#MEX        OFF
#INLINE C_GLOBAL
  extern double kppref_sun_override;
  extern int kppref_sun_ulps;
#ENDINLINE
#INLINE C_RCONST
  if (kppref_sun_override >= 0.0) SUN = kppref_sun_override;
  if (kppref_sun_ulps > 0) SUN = nextafter(SUN, 2.0);
  if (kppref_sun_ulps < 0) SUN = nextafter(SUN, -1.0);
#ENDINLINE
EOF
  if [ "$mech" = "mcm_isoprene" ]; then echo "#INCLUDE    mcm_isoprene_c.eqn" >> "$ds/$mech.kpp"; fi
  (cd "$ds" && KPP_HOME="$KPP_REF" "$OUT/kpp" "$mech.kpp" > kpp.log 2>&1) || {
    echo "build_ref: kpp ($integ) failed for $mech" >&2; tail -20 "$ds/kpp.log" >&2; exit 1; }
  local srcs=() others=() f
  for f in "$ds/${mech}"_*.c; do
    case "$f" in *_mex_*) ;; *) srcs+=("$f") ;; esac
  done
  "$CC" -O -w -fPIC -shared -I"$ds" "${srcs[@]}" -lm -o "$ds/lib${prefix}_${mech}.so"
  "$CC" -O3 -march=x86-64-v3 -ffp-contract=fast -w -fPIC -shared -I"$ds" "${srcs[@]}" -lm \
    -o "$ds/lib${prefix}_${mech}_O3.so"
  for f in "${srcs[@]}"; do
    case "$f" in *_Integrator.c|*_Rates.c) ;; *) others+=("$f") ;; esac
  done
  "$CC" -O -w -fPIC -c -include "$HERE/refkpp/pow_knob.h" -I"$ds" "$ds/${mech}_Integrator.c" -o "$ds/integrator_pw.o"
  "$CC" -O -w -fPIC -c -include "$HERE/refkpp/cos_knob.h" -I"$ds" "$ds/${mech}_Rates.c" -o "$ds/rates_pw.o"
  "$CC" -O -w -fPIC -shared -I"$ds" "${others[@]}" "$ds/integrator_pw.o" "$ds/rates_pw.o" -lm \
    -o "$ds/lib${prefix}_${mech}_pw.so"
  echo "build_ref: $mech ($integ) -> $ds/lib${prefix}_${mech}.so"
}

# A mechanism whose outputs were built from the same oracle sources (this
# script, refkpp/, ros_oracle.c, the MCM translator) is left as it is.
SRC_KEY="$(cat "$HERE/build_ref.sh" "$HERE"/refkpp/*.c "$HERE"/refkpp/*.h "$FRONT/frontend.c" "$HERE/ros_oracle.c" \
  "$HERE"/../kpp_b200/gen/mcm.py "$HERE"/../kpp_b200/gen/fortran.py | sha256sum | cut -d' ' -f1)"

for mech in "${MECHS[@]}"; do
  d="$OUT/$mech"
  if [ -f "$OUT/$mech.stamp" ] && [ "$(cat "$OUT/$mech.stamp")" = "$SRC_KEY" ]; then
    echo "build_ref: $mech up to date"
    continue
  fi
  rm -f "$OUT/$mech.stamp"
  rm -rf "$d"
  mkdir -p "$d"
  # The wrapper selects the C language, the reference Rosenbrock integrator and
  # the batch driver.  C_GLOBAL/C_RCONST add the optional per-cell SUN of the
  # batch driver: Update_RCONST runs the C_RCONST block before the rate
  # assignments (src/gen.c:2420-2435), after FunTemplate called Update_SUN.
  # MCM isoprene: KPP ships it for Fortran 90 only; the mechanism is read from
  # the C translation that the kpp_b200 build makes from examples/mcm
  # (kpp_b200/gen/mcm.py), the same file kppcu reads.
  model="#MODEL      $mech"
  extras="#HESSIAN    ON
#STOICMAT   ON"
  if [ "$mech" = "mcm_isoprene" ]; then
    (cd "$HERE/.." && python -m kpp_b200.gen.mcm --home "$KPP_REF" --out "$d" > /dev/null)
    model=""
    extras="#HESSIAN    OFF
#STOICMAT   OFF"
  fi
  cat > "$d/$mech.kpp" <<EOF
$model
#LANGUAGE   C
#DOUBLE     ON
#INTEGRATOR rosenbrock
#DRIVER     $HERE/refkpp/batch_driver
#JACOBIAN   SPARSE_LU_ROW
$extras
#MEX        OFF
#INLINE C_GLOBAL
  extern double kppref_sun_override;
  extern int kppref_sun_ulps;
#ENDINLINE
#INLINE C_RCONST
  if (kppref_sun_override >= 0.0) SUN = kppref_sun_override;
  if (kppref_sun_ulps > 0) SUN = nextafter(SUN, 2.0);
  if (kppref_sun_ulps < 0) SUN = nextafter(SUN, -1.0);
#ENDINLINE
EOF
  if [ "$mech" = "mcm_isoprene" ]; then echo "#INCLUDE    mcm_isoprene_c.eqn" >> "$d/$mech.kpp"; fi
  (cd "$d" && KPP_HOME="$KPP_REF" "$OUT/kpp" "$mech.kpp" > kpp.log 2>&1) || {
    echo "build_ref: kpp failed for $mech" >&2; tail -20 "$d/kpp.log" >&2; exit 1; }
  srcs=()
  for f in "$d/${mech}"_*.c; do
    case "$f" in *_mex_*) ;; *) srcs+=("$f") ;; esac
  done
  inc=(-include "$d/${mech}_Parameters.h" -include "$d/${mech}_Global.h" -include "$d/${mech}_Sparse.h")
  "$CC" -O -Wall -w -fPIC -shared -I"$d" "${srcs[@]}" \
    -x c "$HERE/ros_oracle.c" "${inc[@]}" -lm -o "$d/libkppref_${mech}.so"
  "$CC" -O3 -march=x86-64-v3 -ffp-contract=fast -w -fPIC -shared -I"$d" "${srcs[@]}" \
    -x c "$HERE/ros_oracle.c" "${inc[@]}" -lm -o "$d/libkppref_${mech}_O3.so"
  if [ "$mech" != "mcm_isoprene" ]; then
    # Update_SUN's cos() through the driver's kppref_cos (refkpp/cos_knob.h),
    # which can move each result one ulp (MCM takes SUN per cell: no cosine)
    others=()
    for f in "${srcs[@]}"; do
      case "$f" in *_Rates.c) ;; *) others+=("$f") ;; esac
    done
    "$CC" -O -w -fPIC -c -include "$HERE/refkpp/cos_knob.h" -I"$d" "$d/${mech}_Rates.c" -o "$d/rates_cs.o"
    "$CC" -O -w -fPIC -shared -I"$d" "${others[@]}" "$d/rates_cs.o" \
      -x c "$HERE/ros_oracle.c" "${inc[@]}" -lm -o "$d/libkppref_${mech}_cs.so"
  fi
  echo "build_ref: $mech -> $d/libkppref_${mech}.so"

  # the same model with the reference SDIRK (int/sdirk.c) and Runge-Kutta
  # (int/runge_kutta.c) integrators and their batch drivers, for those
  # entries' parity tests
  build_integrator_model "$mech" sdirk batch_driver_sdirk sdirk kppsd
  build_integrator_model "$mech" runge_kutta batch_driver_rk rk kpprk
  # and with the reference Rosenbrock adjoint (int/rosenbrock_adj.c), which
  # needs the generated Hessian (not for MCM: its Hessian is not built)
  if [ "$mech" != "mcm_isoprene" ]; then
    build_integrator_model "$mech" rosenbrock_adj batch_driver_adj adj kppadj ON
  fi
  echo "$SRC_KEY" > "$OUT/$mech.stamp"
done
