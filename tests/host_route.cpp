// Host build of the device code that KPP's own generator writes with
// #LANGUAGE CUDA (kpp_b200/kppgen; test infrastructure): the device qualifiers
// removed and the host libm, so that tests compare its Update_RCONST, Fun,
// Jac_SP, KppDecomp and KppSolve with the reference's generated C functions
// and with kppcu's code bit for bit on the CPU.
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
#include ROUTE_INCLUDES

namespace {
struct Species {
  const double* var;
  const double* fix;
  int nvar;
  double operator[](int i) const { return i < nvar ? var[i] : fix[i - nvar]; }
};
}  // namespace

extern "C" {

// sun < 0: SUN from Update_SUN(t) (util/UpdateSun.c), as the reference computes it
void route_rates(int nvar, double temp, double cfactor, double sun, double t, const double* var,
                 const double* fix, double* rconst) {
  const double s = sun >= 0.0 ? sun : kpp_update_sun(t);
  Update_RCONST(rconst, t, temp, cfactor, s, Species{var, fix, nvar});
}

void route_fun(const double* var, const double* fix, const double* rconst, double* vdot) {
  Fun(var, fix, rconst, vdot);
}

void route_jac(const double* var, const double* fix, const double* rconst, double* jvs) {
  Jac_SP(var, fix, rconst, jvs);
}

int route_decomp(double* jvs) { return KppDecomp(jvs); }

void route_solve(const double* jvs, double* x) { KppSolve(jvs, x); }

}  // extern "C"
