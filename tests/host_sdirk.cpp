// Host build of the SDIRK integrator of kpp_b200 (test infrastructure).
//
// kpp_sdirk.cuh and the per-cell definitions it uses (kpp_cell.cuh) are CUDA
// device code; compiled here as plain C++ (device qualifiers removed, host
// libm) on the mechanism code kppcu generated, the integrator can be compared
// with the reference's own C SDIRK on the CPU, where both use the same libm
// and compiler: any difference is then an error of the restatement, not a
// math-library ulp.
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
#define __constant__
#include <cmath>
#include <memory>
using std::cos;
using std::exp;
using std::fma;
using std::log10;
using std::pow;
using std::rint;
using std::sqrt;
using std::fabs;
using std::fmod;
using std::frexp;
using std::isinf;
using std::ldexp;
using std::trunc;
#define KPP_SUN_COS cos
#define KPP_POW pow
#include "kpp_ratelaws.cuh"
#include KPP_MECH_HEADER

// The reference's SQRT is pow(x, 0.5) (int/sdirk.c:4); the device computes
// the correctly rounded sqrt, which glibc's pow(x, 0.5) misses by an ulp for
// rare arguments.  The host build calls pow as the reference does, so that
// the comparison is exact.
#define sqrt(x) pow((x), 0.5)
namespace kpp_b200_impl {
#include "kpp_cell.cuh"
#include "kpp_sdirk.cuh"
}  // namespace kpp_b200_impl

using namespace kpp_b200_impl;

extern "C" {

// Cells [0, ncells) from tstart[c] to tend[c], as kpp_b200_sdirk does on the
// device: the same arrays and layouts (include/kpp_b200.h).
int host_sdirk_integrate(int ncells, int ld, double* var, const double* fix, const double* temp,
                         const double* cfactor, const double* sun, const double* tstart,
                         const double* tend, const double* atol, const double* rtol,
                         const int* icntrl, const double* rcntrl, int* istatus, double* rstatus,
                         int* ierr) {
  auto w = std::make_unique<sdirk::Work>(nullptr, 0L);
  const int nt = icntrl[1] == 0 ? NVAR : 1;
  std::unique_ptr<double[]> at(new double[nt]), rt(new double[nt]);
  for (int i = 0; i < nt; i++) { at[i] = atol[i]; rt[i] = rtol[i]; }
  for (int cell = 0; cell < ncells; cell++) {
    CellEnv env;
    env.temp = temp[cell];
    env.cfactor = cfactor ? cfactor[cell] : KPP_CFACTOR;
    env.sun_fixed = sun ? sun[cell] : -1.0;
    for (int i = 0; i < NFIX; i++) env.fix[i] = (i < NFIX_TRUE) ? fix[(long)i * ld + cell] : 0.0;
    for (int i = 0; i < NVAR; i++) w->y[i] = var[(long)i * ld + cell];
    Stats st = {0, 0, 0, 0, 0, 0, 0, 0};
    double rst[3] = {0.0, 0.0, 0.0};
    ierr[cell] = sdirk::sdirk_cell(env, *w, tstart[cell], tend[cell], at.get(), rt.get(), icntrl,
                                   rcntrl, rst, st);
    for (int i = 0; i < NVAR; i++) var[(long)i * ld + cell] = w->y[i];
    const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
    for (int i = 0; i < 8; i++) istatus[(long)i * ld + cell] = sv[i];
    for (int i = 0; i < 3; i++) rstatus[(long)i * ld + cell] = rst[i];
  }
  return 0;
}

}  // extern "C"
