// Host build of kppcu's generated mechanism code (test infrastructure).
//
// The generated header is CUDA device code; compiled here as plain C++ for
// the host (device qualifiers removed, host libm), so tests can compare the
// emitted arithmetic against the reference's own generated C functions on
// the CPU, where both use the same libm and compiler: any difference is then
// an emitter error, not a math-library ulp.
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
#define __constant__
#include <cmath>
using std::cos;
using std::exp;
using std::fma;
using std::log10;
using std::pow;
using std::rint;
using std::fabs;
using std::fmod;
using std::frexp;
using std::isinf;
using std::ldexp;
using std::trunc;
using std::sqrt;
#define KPP_SUN_COS cos
#define KPP_POW pow
#include "kpp_ratelaws.cuh"

// the device cosine of Update_SUN, for its own test
extern "C" double host_cos_cr(double x) { return kpp_cos_cr(x); }
// the device pow of the integrators' controllers, for its own test
extern "C" double host_pow_cr(double x, double y) { return kpp_pow_cr(x, y); }
#include KPP_MECH_HEADER
#ifdef KPP_ADJ_HEADER
#include KPP_ADJ_HEADER
#endif

extern "C" {

void host_rates(double temp, double cfactor, double sun, double t, const double* var,
                const double* fix, double* rconst) {
  double s = sun >= 0.0 ? sun : kpp_update_sun(t);
  kpp_update_rconst(rconst, t, temp, cfactor, s, var, fix);
}

void host_fun(const double* var, const double* fix, const double* rconst, double* vdot) {
  double a[KPP_NREACT > 0 ? KPP_NREACT : 1];
  kpp_fun(var, fix, rconst, vdot, a);
}

void host_jac(const double* var, const double* fix, const double* rconst, double* jvs) {
  double b[KPP_NJAC_TMP];
  kpp_jac_sp<false>(var, fix, rconst, jvs, b);
}

int host_decomp(double* jvs) {
  double w[KPP_NVAR];  // work row of the loop-form LU of large mechanisms
  return kpp_decomp(jvs, w);
}

void host_solve(const double* jvs, double* x) { kpp_solve(jvs, x); }

#ifdef KPP_ADJ_HEADER
void host_jac_sp_vec(const double* jvs, const double* uv, double* juv) {
  kpp_jac_sp_vec(jvs, uv, juv);
}

void host_jactr_sp_vec(const double* jvs, const double* uv, double* jtuv) {
  kpp_jactr_sp_vec(jvs, uv, jtuv);
}

void host_solve_tr(const double* jvs, const double* x, double* xx) { kpp_solve_tr(jvs, x, xx); }
#endif

}
