// Host build of kpp_b200's Rosenbrock discrete adjoint (test infrastructure).
//
// kpp_adj_int.cuh is CUDA device code over the mechanism functions that KPP's
// own generator writes with #LANGUAGE CUDA and #HESSIAN ON (kpp_b200/kppgen),
// on the sizes and tables of kppcu's header (built with
// KPP_EXTERNAL_ARITHMETIC, as the generator-route library is).  Compiled here
// as plain C++ (device qualifiers removed, host libm), the adjoint can be
// compared with the reference's own C RosenbrockADJ (int/rosenbrock_adj.c)
// on the CPU bit for bit.
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
using std::fabs;
using std::fmod;
using std::frexp;
using std::isinf;
using std::ldexp;
using std::trunc;
using std::sqrt;
#define KPP_SUN_COS cos
#define KPP_POW pow
#define KPP_EXTERNAL_ARITHMETIC
#include "kpp_ratelaws.cuh"
#include KPP_MECH_HEADER
#include ROUTE_INCLUDES
#include "route_adapter.cuh"
namespace kpp_b200_impl {
#include "kpp_cell.cuh"
#include "kpp_adj_int.cuh"
}  // namespace kpp_b200_impl

using namespace kpp_b200_impl;

extern "C" {

// Cells [0, ncells) from tstart[c] to tend[c] as kpp_b200_rosenbrock_adj
// does on the device, with the same arrays and layouts: var [NVAR][ld],
// lambda [nadj * NVAR][ld] (adjoint m's entry i in row m * NVAR + i), in
// place; istatus [8][ld] = ISTATUS[1..8], rstatus [3][ld] = RSTATUS[1..3].
int host_adj_integrate(int ncells, int ld, double* var, const double* fix, const double* temp,
                       const double* cfactor, const double* sun, const double* tstart,
                       const double* tend, const double* atol, const double* rtol, int nadj,
                       double* lambda, const int* icntrl, const double* rcntrl, int bufsize,
                       int* istatus, double* rstatus, int* ierr) {
  const kpp_adj::AdjLayout L = kpp_adj::adj_layout(nadj, bufsize, icntrl[7] != 0);
  std::unique_ptr<double[]> work(new double[L.total]());
  for (int cell = 0; cell < ncells; cell++) {
    CellEnv env;
    env.temp = temp[cell];
    env.cfactor = cfactor ? cfactor[cell] : KPP_CFACTOR;
    env.sun_fixed = sun ? sun[cell] : -1.0;
    for (int i = 0; i < NFIX; i++) env.fix[i] = (i < NFIX_TRUE) ? fix[(long)i * ld + cell] : 0.0;
    kpp_adj::AdjStatus st;
    ierr[cell] = kpp_adj::rosenbrock_adj_cell(
        env, icntrl, rcntrl, atol, rtol, tstart[cell], tend[cell], kpp_adj::Col{var + cell, ld},
        kpp_adj::Col{lambda + cell, ld}, nadj, bufsize, kpp_adj::Col{work.get(), 1}, st);
    const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
    for (int i = 0; i < 8; i++) istatus[(long)i * ld + cell] = sv[i];
    rstatus[cell] = st.texit;
    rstatus[(long)ld + cell] = st.hexit;
    rstatus[2L * ld + cell] = st.hnew;
  }
  return 0;
}

}  // extern "C"
