// The device code that KPP's own generator writes with #LANGUAGE CUDA
// (kpp_b200/kppgen/code_cuda.c), behind the interface kpp_b200's kernels call
// in place of kppcu's functions: rate constants, Fun, Jac_SP, the diagonal
// shift of the Rosenbrock matrix, KppDecomp and KppSolve.  Included by
// kpp_rosenbrock.cu after the generated route_includes.h and the mechanism
// header written by kppcu with KPP_EXTERNAL_ARITHMETIC, which supplies
// everything else (sizes, species, tables, rate classes, the adjoint
// products, the complex LU).
#pragma once

// All species of one cell, variable then fixed, for Update_RCONST's C.
template <class TV, class TF>
struct KppRouteSpecies {
  const TV& var;
  const TF& fix;
  __device__ __forceinline__ double operator[](int i) const {
    return i < KPP_NVAR ? var[i] : fix[i - KPP_NVAR];
  }
};

// Every rate constant: the generator's Update_RCONST recomputes all of them,
// so each of kppcu's dependence classes (static, SUN, dynamic) is served by a
// full evaluation with the same inputs, which gives the same values.
template <class TR, class TV, class TF>
__device__ __forceinline__ void kpp_update_rconst(TR& RCONST, const double TIME, const double TEMP,
                                                  const double CFACTOR, double SUN, const TV& VAR,
                                                  const TF& FIX) {
  Update_RCONST(RCONST, TIME, TEMP, CFACTOR, SUN, KppRouteSpecies<TV, TF>{VAR, FIX});
}
template <class TR, class TV, class TF>
__device__ __forceinline__ void kpp_rconst_static(TR& RCONST, const double TIME, const double TEMP,
                                                  const double CFACTOR, double SUN, const TV& VAR,
                                                  const TF& FIX) {
  kpp_update_rconst(RCONST, TIME, TEMP, CFACTOR, SUN, VAR, FIX);
}
template <class TR, class TV, class TF>
__device__ __forceinline__ void kpp_rconst_sun(TR& RCONST, const double TIME, const double TEMP,
                                               const double CFACTOR, double SUN, const TV& VAR,
                                               const TF& FIX) {
  kpp_update_rconst(RCONST, TIME, TEMP, CFACTOR, SUN, VAR, FIX);
}
template <class TR, class TV, class TF>
__device__ __forceinline__ void kpp_rconst_dynamic(TR& RCONST, const double TIME, const double TEMP,
                                                   const double CFACTOR, double SUN, const TV& VAR,
                                                   const TF& FIX) {
  kpp_update_rconst(RCONST, TIME, TEMP, CFACTOR, SUN, VAR, FIX);
}

template <class TV, class TF, class TR, class TO, class TA>
__device__ __forceinline__ void kpp_fun(const TV& V, const TF& F, const TR& RCT, TO& Vdot, TA&) {
  Fun(V, F, RCT, Vdot);
}

// NEG: the Rosenbrock matrix's -Jac; negating each entry of the generator's
// Jac_SP gives the same bits as evaluating the negated sums.
template <bool NEG, class TV, class TF, class TR, class TJ, class TB>
__device__ __forceinline__ void kpp_jac_sp(const TV& V, const TF& F, const TR& RCT, TJ& JVS, TB&) {
  Jac_SP(V, F, RCT, JVS);
  if (NEG)
    for (int n = 0; n < KPP_LU_NONZERO; n++) JVS[n] = -JVS[n];
}

template <class TJ>
__device__ __forceinline__ void kpp_add_diagonal(TJ& JVS, const double v) {
  for (int i = 0; i < KPP_NVAR; i++) JVS[LU_DIAG[i]] = JVS[LU_DIAG[i]] + v;
}

template <class TJ, class TW>
__device__ __forceinline__ int kpp_decomp(TJ& JVS, TW&) {
  return KppDecomp(JVS);
}

template <class TJ, class TX>
__device__ __forceinline__ void kpp_solve(const TJ& JVS, TX& X) {
  KppSolve(JVS, X);
}
