// Batched Rosenbrock integrator for KPP mechanisms on B200 (sm_100a), and the
// C ABI of include/kpp_b200.h.
//
// Built once per mechanism: KPP_MECH_HEADER names the kppcu output for it.
//
// Design
//   * One grid cell per thread.  Cells are independent stiff ODE systems, so
//     a cell never waits on another; the kernel is a plain data-parallel map.
//   * Cell state lives in registers and thread-local memory; the batched
//     inputs/outputs are structure-of-arrays with the cell index fastest, so
//     every load/store of a warp is one coalesced 256-byte access.
//   * The mechanism (rates, Fun, Jac_SP, LU, solves) is fully unrolled device
//     code from kppcu; the method (tableau) is a template parameter, so stage
//     loops unroll and zero coefficients disappear at compile time.
//   * Arithmetic follows int/rosenbrock.c operation for operation; the
//     library is built with --fmad=false so nothing is contracted into FMAs.
//     Results then match the reference C code up to the last-ulp differences
//     of exp/pow/log10/cos between the CUDA math library and the host libm.
//
// Reference: int/rosenbrock.c (Rosenbrock :137-446, RosenbrockIntegrator
// :450-627, ros_ErrorNorm :632-659, ros_FunTimeDerivative :663-682,
// ros_PrepareMatrix :686-737, tableaux :779-1222, Fun/JacTemplate
// :1257-1296), util/blas.c (WAXPY skips alpha == 0, :51-82), util/sutil.c.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <atomic>
#include <mutex>

#include "../../include/kpp_b200.h"
#include "kpp_ratelaws.cuh"
#include KPP_MECH_HEADER
#ifdef KPP_ROUTE_INCLUDE
// The arithmetic written by KPP's own generator (#LANGUAGE CUDA,
// kpp_b200/kppgen) in place of kppcu's; the warp-per-cell kernel, which runs
// on kppcu's schedules, is left out of such a build.
#include KPP_ROUTE_INCLUDE
#include "route_adapter.cuh"
#undef KPP_COOP
#define KPP_COOP 0
#endif
#if KPP_PART == 7
#include KPP_CMPLX_HEADER
#endif
#if KPP_PART == 0
#include KPP_ADJ_HEADER
#endif

// Translation-unit split (the build compiles this file once per part, in
// parallel): KPP_PART 1..5 holds the kernel of Rosenbrock method 1..5 and its
// launcher; KPP_PART 0 holds everything else and the C ABI.
#ifndef KPP_PART
#define KPP_PART 0
#endif
// Default of the automatic kernel choice's cell limit (kpp_b200_set_auto_warp_cells).
#ifndef KPP_COOP_MAX_CELLS
#if defined(KPP_SCRATCH)
// saprc99 on B200: the warp-per-cell kernel measured faster than the
// thread-per-cell one at every batch size from 2^11 to 2^20 cells
#define KPP_COOP_MAX_CELLS 0x7fffffff
#else
#define KPP_COOP_MAX_CELLS 0
#endif
#endif

namespace kpp_b200_impl {
#include "kpp_cell.cuh"

// ros_ErrorNorm (int/rosenbrock.c:632-659); SQRT(x) of the reference is
// pow(x, 0.5), computed here as the correctly rounded sqrt.
template <class TA, class TB, class TC>
__device__ __forceinline__ double error_norm(const TA& y, const TB& ynew, const TC& yerr,
                                             const double* atol, const double* rtol,
                                             bool vectortol) {
  double err = 0.0;
  const double a0 = atol[0], r0 = rtol[0];
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) {
    double ymax = ros_max(ros_abs(y[i]), ros_abs(ynew[i]));
    double scale = vectortol ? (atol[i] + rtol[i] * ymax) : (a0 + r0 * ymax);
    err = err + (yerr[i] * yerr[i]) / (scale * scale);
  }
  return sqrt(err / (double)NVAR);
}

// ros_PrepareMatrix (int/rosenbrock.c:686-737): Ghimj = -Jac0 + 1/(H*gam) I,
// LU factorise; halve H on a singular factorisation, give up after 5.
// Instead of keeping Jac0 the negated Jacobian is evaluated straight into
// Ghimj at time t (rates at t are in w.rconst); a second attempt evaluates it
// again from the same inputs, which reproduces Jac0 exactly.
template <class W>
__device__ __forceinline__ bool prepare_matrix(const CellEnv& env, double t, double& h,
                                               int direction, double gam, W& w, Stats& st) {
  int nconsecutive = 0;
  for (;;) {
    kpp_jac_sp<true>(w.y, env.fix, w.rconst, w.jvs, w.b);
    double ghinv = 1.0 / (direction * h * gam);
    kpp_add_diagonal(w.jvs, ghinv);
    int ising = kpp_decomp(w.jvs, w.yerr);  // Yerr is free here: the work row
    st.ndec++;
    if (ising == 0) return false;
    st.nsng++;
    nconsecutive++;
    if (nconsecutive <= 5) h = h * 0.5;
    else return true;
  }
}

// Controls of one Rosenbrock call after validation and defaults.
struct RosControls {
  bool autonomous, vectortol;
  int max_no_steps;
  double hmin, hmax, hstart, facmin, facmax, facrej, facsafe;
  const double *atol, *rtol;
};

// Rosenbrock (int/rosenbrock.c:137-446): validation and defaults of a call
// over [tstart, tend] whose Hstart is rpar2 (RPAR[2], or the cell's own).
// Returns 0, or the IERR (-1..-5) of the first rejected control in the
// reference's order of checks.
__device__ __forceinline__ int ros_controls(const LaunchArgs& a, double tstart, double tend,
                                            double rpar2, RosControls& c) {
  const int* ipar = a.ipar;
  const double* rpar = a.rpar;
  c.atol = a.atol;
  c.rtol = a.rtol;
  c.autonomous = !(ipar[0] == 0);
  c.vectortol = (ipar[1] == 0);
  const int uplimtol = c.vectortol ? NVAR : 1;
  c.max_no_steps = (ipar[2] == 0) ? 100000 : ipar[2];
  if (c.max_no_steps < 0) return KPP_B200_IERR_MAXSTEPS_BAD;
  if ((ipar[3] < 1) || (ipar[3] > 5)) return KPP_B200_IERR_METHOD;
  c.hmin = rpar[0];
  if (rpar[0] < 0.0) return KPP_B200_IERR_HBOUNDS;
  c.hmax = (rpar[1] == 0.0) ? ros_abs_diff(tend, tstart)
                            : ros_min(ros_abs(rpar[1]), ros_abs_diff(tend, tstart));
  if (rpar[1] < 0.0) return KPP_B200_IERR_HBOUNDS;
  c.hstart = (rpar2 == 0.0) ? ros_max(c.hmin, kDeltaMin)
                            : ros_min(ros_abs(rpar2), ros_abs_diff(tend, tstart));
  if (rpar2 < 0.0) return KPP_B200_IERR_HBOUNDS;
  c.facmin = (rpar[3] == 0.0) ? 0.2 : rpar[3];
  if (rpar[3] < 0.0) return KPP_B200_IERR_FACTORS;
  c.facmax = (rpar[4] == 0.0) ? 6.0 : rpar[4];
  if (rpar[4] < 0.0) return KPP_B200_IERR_FACTORS;
  c.facrej = (rpar[5] == 0.0) ? 0.1 : rpar[5];
  if (rpar[5] < 0.0) return KPP_B200_IERR_FACTORS;
  c.facsafe = (rpar[6] == 0.0) ? 0.9 : rpar[6];
  if (rpar[6] < 0.0) return KPP_B200_IERR_FACTORS;
  for (int i = 0; i < uplimtol; i++)
    if ((c.atol[i] <= 0.0) || (c.rtol[i] <= 10.0 * kRoundoff) || (c.rtol[i] >= 1.0))
      return KPP_B200_IERR_TOLERANCES;
  return 0;
}

// RosenbrockIntegrator's state (int/rosenbrock.c:450-627) between its steps.
struct RosState {
  double t, tend, h, hexit;
  int direction;
  bool reject_last, reject_more, varying;
};

// Start of RosenbrockIntegrator (:450-470); w.y holds the cell state.
template <class W>
__device__ __forceinline__ void ros_begin(const CellEnv& env, W& w, const RosControls& c,
                                          double tstart, double tend, RosState& s) {
  s.t = tstart;
  s.tend = tend;
  s.hexit = 0.0;
  s.h = ros_min(c.hstart, c.hmax);
  if (ros_abs(s.h) <= 10.0 * kRoundoff) s.h = kDeltaMin;
  s.direction = (tend >= tstart) ? +1 : -1;
  s.reject_last = false;
  s.reject_more = false;
  s.varying = rates_vary<W>(env);
  rates_once(env, s.t, w);
}

// Head of the time loop (:471-529): KPP_B200_IERR_SUCCESS when the loop is
// done, -6 / -7 when the call fails, else 0 after Fcn0 = Fun(T, Y), dF/dT
// and the Jacobian count (each attempt's prepare_matrix evaluates the
// Jacobian itself).
template <class W>
__device__ __forceinline__ int ros_step_head(const CellEnv& env, W& w, const RosControls& c,
                                             RosState& s, Stats& st) {
  if (!(((s.direction > 0) && ((s.t - s.tend) + kRoundoff <= 0.0)) ||
        ((s.direction < 0) && ((s.tend - s.t) + kRoundoff <= 0.0))))
    return KPP_B200_IERR_SUCCESS;
  if (st.nstp > c.max_no_steps) return KPP_B200_IERR_TOO_MANY_STEPS;
  if (((s.t + 0.1 * s.h) == s.t) || (s.h <= kRoundoff)) return KPP_B200_IERR_STEP_TOO_SMALL;
  s.hexit = s.h;
  s.h = ros_min(s.h, ros_abs_diff(s.tend, s.t));

  // FunTemplate(T, Y, Fcn0)
  rates_at(env, s.t, w);
  kpp_fun(w.y, env.fix, w.rconst, w.fcn0, w.a);
  st.nfun++;
  if (!c.autonomous) {
    // ros_FunTimeDerivative (:663-682): dFdT = (Fun(T+Delta) - Fcn0)/Delta
    double delta = sqrt(kRoundoff) * ros_max(kDeltaMin, ros_abs(s.t));
    if (s.varying) {
      rates_at(env, s.t + delta, w);
      kpp_fun(w.y, env.fix, w.rconst, w.dfdt, w.a);
      rates_at(env, s.t, w);  // JacTemplate(T) below sees the rates at T
    } else {
      // Fun(T+Delta) would see the same rates and state: Fcn0 again
      copy(w.fcn0, w.dfdt);
    }
    st.nfun++;
    axpy(-1.0, w.fcn0, w.dfdt);
    double inv = 1.0 / delta;
    if (inv != 1.0) {
#pragma unroll 4
      for (int i = 0; i < NVAR; i++) w.dfdt[i] = inv * w.dfdt[i];
    }
  }
  st.njac++;  // JacTemplate(T, Y, Jac0), evaluated inside prepare_matrix
  return 0;
}

// One attempt of the UntilAccepted loop (:531-611): 1 when the step is
// accepted (T and Y advanced), 0 when it is rejected (H reduced: the next
// attempt follows), or KPP_B200_IERR_SINGULAR.  `retry` is false for the
// first attempt of a step.
template <int METHOD, class W>
__device__ __forceinline__ int ros_attempt(const CellEnv& env, W& w, const RosControls& c,
                                           RosState& s, bool& retry, Stats& st) {
  constexpr Tableau tab = make_tableau(METHOD);
  constexpr int S = tab.S;
  const int direction = s.direction;
  if (retry && s.varying) rates_at(env, s.t, w);  // stages moved the rates to Tau
  retry = true;
  if (prepare_matrix(env, s.t, s.h, direction, tab.Gamma[0], w, st))
    return KPP_B200_IERR_SINGULAR;
  const double h = s.h;
#pragma unroll
  for (int j = 0; j < S; j++) {
    if (j == 0) {
      copy(w.fcn0, w.fcn);
    } else if (tab.NewF[j]) {
      copy(w.y, w.ynew);
#pragma unroll
      for (int i = 0; i < j; i++) axpy(tab.A[j * (j - 1) / 2 + i], w.k[i], w.ynew);
      double tau = s.t + tab.Alpha[j] * direction * h;
      if (s.varying) rates_at(env, tau, w);
      kpp_fun(w.ynew, env.fix, w.rconst, w.fcn, w.a);
      st.nfun++;
    }
    copy(w.fcn, w.k[j]);
#pragma unroll
    for (int i = 0; i < j; i++) {
      double hc = tab.C[j * (j - 1) / 2 + i] / (direction * h);
      axpy(hc, w.k[i], w.k[j]);
    }
    if ((!c.autonomous) && (tab.Gamma[j] != 0.0)) {
      double hg = direction * h * tab.Gamma[j];
      axpy(hg, w.dfdt, w.k[j]);
    }
    kpp_solve(w.jvs, w.k[j]);
    st.nsol++;
  }

  copy(w.y, w.ynew);
#pragma unroll
  for (int j = 0; j < S; j++) axpy(tab.M[j], w.k[j], w.ynew);
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) w.yerr[i] = 0.0;
#pragma unroll
  for (int j = 0; j < S; j++) axpy(tab.E[j], w.k[j], w.yerr);
  double err = error_norm(w.y, w.ynew, w.yerr, c.atol, c.rtol, c.vectortol);

  double fac = ros_min(c.facmax, ros_max(c.facmin, c.facsafe / KPP_POW(err, 1.0 / tab.ELO)));
  double hnew = h * fac;

  st.nstp++;
  if ((err <= 1.0) || (h <= c.hmin)) {
    st.nacc++;
    copy(w.ynew, w.y);
    s.t += direction * h;
    hnew = ros_max(c.hmin, ros_min(hnew, c.hmax));
    if (s.reject_last) hnew = ros_min(hnew, h);
    s.reject_last = false;
    s.reject_more = false;
    s.h = hnew;
    return 1;
  }
  if (st.nacc >= 1) st.nrej++;
  if (s.reject_more) hnew = h * c.facrej;
  s.reject_more = s.reject_last;
  s.reject_last = true;
  s.h = hnew;
  return 0;
}

// RosenbrockIntegrator (int/rosenbrock.c:450-627) for one cell; w.y holds
// the cell state in and out.  Returns IERR; Texit, Hexit and the counters.
template <int METHOD, class W>
__device__ int integrate_cell(const CellEnv& env, W& w, const RosControls& c, double tstart,
                              double tend, double& texit, double& hexit, Stats& st) {
  RosState s;
  ros_begin(env, w, c, tstart, tend, s);
  for (;;) {
    const int head = ros_step_head(env, w, c, s, st);
    if (head != 0) {
      texit = s.t;
      hexit = s.hexit;
      return head;
    }
    bool retry = false;
    for (;;) {
      const int r = ros_attempt<METHOD>(env, w, c, s, retry, st);
      if (r == 1) break;
      if (r != 0) {
        texit = s.t;
        hexit = s.hexit;
        return r;
      }
    }
  }
}

// Rosenbrock (int/rosenbrock.c:137-446): validation and defaults, then the
// integrator.  Returns IERR; fills stats/texit/hexit like IPAR/RPAR[10..].
template <int METHOD, class W>
__device__ int rosenbrock_cell(const CellEnv& env, W& w, double tstart, double tend,
                               const LaunchArgs& a, double rpar2, Stats& st, double& texit,
                               double& hexit) {
  RosControls c;
  const int bad = ros_controls(a, tstart, tend, rpar2, c);
  if (bad) return bad;
  return integrate_cell<METHOD>(env, w, c, tstart, tend, texit, hexit, st);
}

__device__ __forceinline__ void load_env(CellEnv& env, const double* temp, const double* cfactor,
                                         const double* sun, const double* fix, long ld, int cell) {
  env.temp = temp[cell];
  env.cfactor = cfactor ? cfactor[cell] : KPP_CFACTOR;
  env.sun_fixed = sun ? sun[cell] : -1.0;
#pragma unroll
  for (int i = 0; i < NFIX; i++) env.fix[i] = (i < NFIX_TRUE) ? fix[i * ld + cell] : 0.0;
}

// Text of the last error of the calling thread (defined in part 0).
extern thread_local char g_last_error[512];

inline int fail(int code, const char* msg) {
  std::snprintf(g_last_error, sizeof g_last_error, "%s", msg);
  return code;
}

inline int cuda_fail(const char* what, cudaError_t e) {
  std::snprintf(g_last_error, sizeof g_last_error, "%s: %s", what, cudaGetErrorString(e));
  return KPP_B200_ECUDA;
}

inline int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? KPP_B200_OK : cuda_fail(what, e);
}

constexpr int kBlock = 128;

// Set-up done once per device: `get` runs f(device) the first time it is
// called with that device current (under a lock, so concurrent first calls
// from several host threads do it once) and returns the value f gave.
struct DeviceOnce {
  std::mutex mu;
  std::map<int, int> value;
  template <class F>
  int get(F f) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    std::lock_guard<std::mutex> lock(mu);
    auto it = value.find(dev);
    if (it == value.end()) it = value.emplace(dev, f(dev)).first;
    return it->second;
  }
};

// Launcher and occupancy of the kernel of method M, defined in part M.
template <int M>
int launch_method(LaunchArgs& a, int grid, cudaStream_t s);
template <int M>
int occupancy_method();
// The warp-per-cell kernel of method M (kpp_coop.cuh).
template <int M>
int launch_method_coop(LaunchArgs& a, cudaStream_t s);
// The SDIRK kernel (KPP_PART 6).
int launch_sdirk(LaunchArgs& a, int grid, cudaStream_t s);

#if KPP_PART >= 1
// Resident blocks per SM the compiler must allow (bounds the registers per
// thread: 65536 / (128 * KPP_MIN_BLOCKS)); 0 leaves the choice to ptxas.
// 8 blocks (64 registers) measured fastest for saprc99 on B200.
#ifndef KPP_MIN_BLOCKS
#define KPP_MIN_BLOCKS 8
#endif

// Integrates one cell: one Rosenbrock call over [tstart, tend], or with
// CHAIN (a.nchain >= 1) the driver loop of drv/general.c:59-76 around
// INTEGRATE (int/rosenbrock.c:94-133): a.nchain calls Rosenbrock(T, T + dt),
// T += dt, each call's Hstart = the previous call's Hexit (STEPMIN), counters
// summed (INTEGRATE's Ns/Na/Nr/Ng), Texit/Hexit of the last call, IERR of the
// first failing call (1 when every call succeeds).  Failing calls do not stop
// the loop, as the reference driver continues after INTEGRATE reports them.
__device__ __forceinline__ void record_call(const LaunchArgs& a, int cell, bool first, int ierr,
                                            const Stats& st, double texit, double hexit) {
  const long ld = a.ld;
  // y is untouched when the controls were rejected (IERR -1..-5); the
  // statistics and Texit/Hexit are then zero, as IPAR/RPAR[10..] stay.
  const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
  if (first) {
    a.ierr[cell] = ierr;
#pragma unroll
    for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] = sv[i];
  } else {
    if (a.ierr[cell] == KPP_B200_IERR_SUCCESS) a.ierr[cell] = ierr;
#pragma unroll
    for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] += sv[i];
  }
  a.rstatus[cell] = texit;
  a.rstatus[ld + cell] = hexit;
}

template <int METHOD, bool CHAIN, class W>
__device__ __forceinline__ void one_call(const LaunchArgs& a, W& w, const CellEnv& env, int cell,
                                         int k, double& t0, double& rpar2) {
  const double t1 = CHAIN ? t0 + a.chain_dt : a.tend[cell];
  Stats st = {0, 0, 0, 0, 0, 0, 0, 0};
  double texit = 0.0, hexit = 0.0;
  const int ierr = rosenbrock_cell<METHOD>(env, w, t0, t1, a, rpar2, st, texit, hexit);
  record_call(a, cell, !CHAIN || k == 0, ierr, st, texit, hexit);
  rpar2 = hexit;  // STEPMIN = RPAR[11]
  t0 = t1;        // TIME += DT
}

// Integrates one cell: one Rosenbrock call over [tstart, tend] (grid-stride
// launch, has = true), or, for the work queue, the driver loop of
// drv/general.c:59-76 around INTEGRATE (int/rosenbrock.c:94-133): a.nchain
// calls Rosenbrock(T, T + dt), T += dt, each call's Hstart = the previous
// call's Hexit (STEPMIN), counters summed (INTEGRATE's Ns/Na/Nr/Ng),
// Texit/Hexit of the last call, IERR of the first failing call (1 when every
// call succeeds).  Failing calls do not stop the loop, as the reference
// driver continues after INTEGRATE reports them.  In the queue form all 32
// lanes of a warp call this together (has = false: no cell, the lane only
// joins the barriers), and a warp barrier after each call starts the lanes'
// next chemistry step together, so the lanes stay in the same phase of the
// integrator instead of drifting apart over the calls.
template <int METHOD, bool CHAIN, class W>
__device__ __forceinline__ void integrate_cell_calls(const LaunchArgs& a, W& w, int cell,
                                                     bool has = true) {
  const long ld = a.ld;
  CellEnv env;
  double t0 = 0.0, rpar2 = 0.0;
  if (has) {
    load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, cell);
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.y[i] = a.var[i * ld + cell];
    t0 = a.tstart[cell];
    rpar2 = a.hstart ? a.hstart[cell] : a.rpar[2];
  }
  if (CHAIN) {
    for (int k = 0; k < a.nchain; k++) {
      if (has) one_call<METHOD, true>(a, w, env, cell, k, t0, rpar2);
      __syncwarp();
    }
  } else {
    one_call<METHOD, false>(a, w, env, cell, 0, t0, rpar2);
  }
  if (has) {
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) a.var[i * ld + cell] = w.y[i];
  }
}

// The lane-granular work queue (a.lane_queue): every lane runs its own
// cell's chained calls as a state machine that advances by one step attempt
// per pass of a loop the 32 lanes make together, and takes the next queue
// position as soon as its cell is done.  The attempts (Jacobian, LU, stages,
// error estimate: most of the work) of all lanes remain one instruction
// stream however far apart the lanes' cells are, so no lane waits for the
// slowest cell of its warp; what one lane does alone (loading a cell,
// starting a call, a step's head: rates and Fun) the others wait for.  Each
// cell's operations are integrate_cell_calls' in the same order, so results
// are bit-identical to the other launches.
template <int METHOD, class W>
__device__ void integrate_refill(const LaunchArgs& a, W& w) {
  enum { kCell, kCall, kHead, kTry };
  const long ld = a.ld;
  CellEnv env;
  RosControls c;
  RosState s;
  Stats st = {0, 0, 0, 0, 0, 0, 0, 0};
  int phase = kCell, cell = 0, k = 0;
  double t0 = 0.0, t1 = 0.0, rpar2 = 0.0;
  bool retry = false;
  for (;;) {
    // this lane's cell and call starts and step heads, until it has an
    // attempt to make
    while (phase != kTry) {
      if (phase == kCell) {
        const int pos = atomicAdd(a.queue, 1);
        if (pos >= a.ncells) return;
        cell = a.order ? a.order[pos] : pos;
        load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, cell);
#pragma unroll 4
        for (int i = 0; i < NVAR; i++) w.y[i] = a.var[i * ld + cell];
        t0 = a.tstart[cell];
        rpar2 = a.hstart ? a.hstart[cell] : a.rpar[2];
        k = 0;
        phase = kCall;
      }
      int end = 0;  // nonzero: the call ends with this IERR
      double texit = 0.0, hexit = 0.0;
      if (phase == kCall) {
        t1 = t0 + a.chain_dt;
        st = {0, 0, 0, 0, 0, 0, 0, 0};
        end = ros_controls(a, t0, t1, rpar2, c);
        if (!end) {
          ros_begin(env, w, c, t0, t1, s);
          phase = kHead;
        }
      }
      if (phase == kHead) {
        end = ros_step_head(env, w, c, s, st);
        if (end) {
          texit = s.t;
          hexit = s.hexit;
        } else {
          retry = false;
          phase = kTry;
        }
      }
      if (end) {
        record_call(a, cell, k == 0, end, st, texit, hexit);
        rpar2 = hexit;  // STEPMIN = RPAR[11]
        t0 = t1;        // TIME += DT
        if (++k < a.nchain) {
          phase = kCall;
        } else {
#pragma unroll 4
          for (int i = 0; i < NVAR; i++) a.var[i * ld + cell] = w.y[i];
          phase = kCell;
        }
      }
    }
    const int r = ros_attempt<METHOD>(env, w, c, s, retry, st);
    if (r == 1) {
      phase = kHead;
    } else if (r != 0) {
      record_call(a, cell, k == 0, r, st, s.t, s.hexit);
      rpar2 = s.hexit;
      t0 = t1;
      if (++k < a.nchain) {
        phase = kCall;
      } else {
#pragma unroll 4
        for (int i = 0; i < NVAR; i++) a.var[i * ld + cell] = w.y[i];
        phase = kCell;
      }
    }
  }
}

// QUEUE = false: one thread slot integrates cells slot, slot + nslots, ...
// (grid-stride), one call each.  QUEUE = true: each warp takes the next 32
// queue positions from the device counter until the queue is empty
// (persistent launch: the grid is the resident thread count) and runs the
// chained calls of each cell.  A queue ordered by decreasing cost hands the
// long cells out first and keeps the 32 cells of a warp of similar cost.
// With a.lane_queue each lane instead takes the next single position as soon
// as its previous cell is done (integrate_refill).
template <int METHOD, bool QUEUE>
__global__ void
#if KPP_MIN_BLOCKS > 0
__launch_bounds__(128, KPP_MIN_BLOCKS)
#else
__launch_bounds__(128)
#endif
rosenbrock_kernel(const LaunchArgs a) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  Work w(a.scratch, a.nslots, slot);
  if (QUEUE && a.lane_queue) {
    integrate_refill<METHOD>(a, w);
  } else if (QUEUE) {
    const int lane = threadIdx.x & 31;
    for (;;) {
      int base = 0;
      if (lane == 0) base = atomicAdd(a.queue, 32);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= a.ncells) break;  // warp-uniform
      const int pos = base + lane;
      const bool has = pos < a.ncells;
      integrate_cell_calls<METHOD, true>(a, w, has ? (a.order ? a.order[pos] : pos) : 0, has);
    }
  } else {
    for (long c = slot; c < a.ncells; c += a.nslots)
      integrate_cell_calls<METHOD, false>(a, w, (int)c);
  }
}


template <int M>
int launch_method(LaunchArgs& a, int grid, cudaStream_t s) {
  // the kernel uses no shared memory: all of it as L1 (a per-device attribute)
  static DeviceOnce carveout;
  carveout.get([](int) {
    cudaFuncSetAttribute(rosenbrock_kernel<M, true>,
                         cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    cudaFuncSetAttribute(rosenbrock_kernel<M, false>,
                         cudaFuncAttributePreferredSharedMemoryCarveout, 0);
    return 1;
  });
  if (a.queue)
    rosenbrock_kernel<M, true><<<grid, kBlock, 0, s>>>(a);
  else
    rosenbrock_kernel<M, false><<<grid, kBlock, 0, s>>>(a);
  return check_launch("rosenbrock_kernel");
}

template <int M>
int occupancy_method() {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rosenbrock_kernel<M, false>, kBlock,
                                                    0) !=
      cudaSuccess)
    per_sm = 1;
  return per_sm;
}

#if KPP_PART <= 5
template int launch_method<KPP_PART>(LaunchArgs&, int, cudaStream_t);
template int occupancy_method<KPP_PART>();
#endif

#if KPP_COOP
#include "kpp_coop.cuh"

// The warp-per-cell kernel of method M: one CTA of W warps per SM (shared
// memory holds the tables and W cells), at most one CTA per W cells.
template <int M>
int launch_method_coop(LaunchArgs& a, cudaStream_t s) {
  constexpr int S = make_tableau(M).S;
  constexpr int W = coop::warps_per_cta<S>();
  constexpr size_t bytes = coop::smem_bytes<S>();
  static_assert(W >= 1, "kppcu only writes tables for cells that fit shared memory");
  static DeviceOnce sms_of;  // SMs of the device, with the kernels' attributes set there
  const int sms = sms_of.get([](int dev) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    if (cudaFuncSetAttribute(coop::kernel<M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes) != cudaSuccess ||
        cudaFuncSetAttribute(coop::kernel<M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes) != cudaSuccess)
      return -1;
    return n;
  });
  if (sms < 1) return fail(KPP_B200_ECUDA, "warp-per-cell kernel: device set-up failed");
  const long want = ((long)a.ncells + W - 1) / W;
  const int grid = (int)(want < sms ? want : sms);
  if (a.queue)
    coop::kernel<M, true><<<grid, 32 * W, bytes, s>>>(a);
  else
    coop::kernel<M, false><<<grid, 32 * W, bytes, s>>>(a);
  return check_launch("warp-per-cell rosenbrock kernel");
}

#if KPP_PART <= 5
template int launch_method_coop<KPP_PART>(LaunchArgs&, cudaStream_t);
#endif
#endif  // KPP_COOP

#if KPP_PART == 6
#include "kpp_sdirk.cuh"

// One thread slot integrates cells slot, slot + nslots, ... with the C SDIRK
// (int/sdirk.c); ICNTRL / RCNTRL travel in ipar / rpar of the launch.
__global__ void
#if KPP_MIN_BLOCKS > 0
__launch_bounds__(128, KPP_MIN_BLOCKS)
#else
__launch_bounds__(128)
#endif
sdirk_kernel(const LaunchArgs a) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long ld = a.ld;
  sdirk::Work w(a.scratch, slot);
  for (long c = slot; c < a.ncells; c += a.nslots) {
    const int cell = (int)c;
    CellEnv env;
    load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, cell);
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.y[i] = a.var[i * ld + cell];
    Stats st = {0, 0, 0, 0, 0, 0, 0, 0};
    double rst[3] = {0.0, 0.0, 0.0};
    const int ierr = sdirk::sdirk_cell(env, w, a.tstart[cell], a.tend[cell], a.atol, a.rtol,
                                       a.ipar, a.rpar, rst, st);
    a.ierr[cell] = ierr;
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) a.var[i * ld + cell] = w.y[i];
    const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
#pragma unroll
    for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] = sv[i];
#pragma unroll
    for (int i = 0; i < 3; i++) a.rstatus[i * ld + cell] = rst[i];
  }
}

int launch_sdirk(LaunchArgs& a, int grid, cudaStream_t s) {
  sdirk_kernel<<<grid, kBlock, 0, s>>>(a);
  return check_launch("sdirk_kernel");
}
#endif  // KPP_PART == 6

#if KPP_PART == 7
#include "kpp_rk.cuh"

// One thread slot integrates cells slot, slot + nslots, ... with the C
// RungeKutta (int/runge_kutta.c); the shared controls and the method table
// come in `c`, RCNTRL in rpar of the launch.
__global__ void
#if KPP_MIN_BLOCKS > 0
__launch_bounds__(128, KPP_MIN_BLOCKS)
#else
__launch_bounds__(128)
#endif
rk_kernel(const LaunchArgs a, const rk::Controls c) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long ld = a.ld;
  rk::Work w(a.scratch, slot);
  for (long cc = slot; cc < a.ncells; cc += a.nslots) {
    const int cell = (int)cc;
    CellEnv env;
    load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, cell);
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.y[i] = a.var[i * ld + cell];
    Stats st = {0, 0, 0, 0, 0, 0, 0, 0};
    double rst[3] = {0.0, 0.0, 0.0};
    const int ierr =
        rk::rk_cell(env, w, c, a.tstart[cell], a.tend[cell], a.rpar, a.atol, a.rtol, rst, st);
    a.ierr[cell] = ierr;
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) a.var[i * ld + cell] = w.y[i];
    const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
#pragma unroll
    for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] = sv[i];
#pragma unroll
    for (int i = 0; i < 3; i++) a.rstatus[i * ld + cell] = rst[i];
  }
}

int launch_rk(LaunchArgs& a, int grid, cudaStream_t s) {
  const rk::Controls c = rk::make_controls(a.ipar, a.rpar);
  rk_kernel<<<grid, kBlock, 0, s>>>(a, c);
  return check_launch("rk_kernel");
}
#endif  // KPP_PART == 7

#if KPP_PART == 8
#include "kpp_adj_int.cuh"

// The Rosenbrock discrete adjoint (kpp_adj_int.cuh), one thread per cell;
// ICNTRL / RCNTRL travel in ipar / rpar of the launch.  Each cell's work
// arrays and trajectory are column `cell` of `work` (element e at
// work[e * ld + cell]), so the threads of a warp touch consecutive words.
__global__ void __launch_bounds__(128) adj_kernel(const LaunchArgs a, double* lambda, int nadj,
                                                  int bufsize, double* work) {
  const long cell = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= a.ncells) return;
  const long ld = a.ld;
  CellEnv env;
  load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, (int)cell);
  kpp_adj::AdjStatus st;
  const int ierr = kpp_adj::rosenbrock_adj_cell(
      env, a.ipar, a.rpar, a.atol, a.rtol, a.tstart[cell], a.tend[cell],
      kpp_adj::Col{a.var + cell, ld}, kpp_adj::Col{lambda + cell, ld}, nadj, bufsize,
      kpp_adj::Col{work + cell, ld}, st);
  a.ierr[cell] = ierr;
  const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
#pragma unroll
  for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] = sv[i];
  a.rstatus[cell] = st.texit;
  a.rstatus[ld + cell] = st.hexit;
  a.rstatus[2 * ld + cell] = st.hnew;
}

int launch_adj(LaunchArgs& a, double* lambda, int nadj, int bufsize, double* work,
               cudaStream_t s) {
  const int grid = (a.ncells + kBlock - 1) / kBlock;
  adj_kernel<<<grid, kBlock, 0, s>>>(a, lambda, nadj, bufsize, work);
  return check_launch("adj_kernel");
}
#endif  // KPP_PART == 8

#else  // KPP_PART == 0

#define KPP_RK_HOST_ONLY
#include "kpp_rk.cuh"
// The Runge-Kutta kernel (KPP_PART 7).
int launch_rk(LaunchArgs& a, int grid, cudaStream_t s);
#if defined(KPP_NHESS)
#include "kpp_adj_int.cuh"
// The Rosenbrock discrete adjoint kernel (KPP_PART 8), in libraries built on
// the generator route with the Hessian.
int launch_adj(LaunchArgs& a, double* lambda, int nadj, int bufsize, double* work,
               cudaStream_t s);
#endif

thread_local char g_last_error[512] = "";

// Which kernel integrates: 0 automatic, 1 thread per cell, 2 warp per cell
// (kpp_coop.cuh).  The warp-per-cell kernel runs only launches whose rate
// constants are fixed for the call; the others always use the thread kernel.
int g_kernel_choice = 0;
// Work-queue granularity of the chained entry's thread-per-cell kernel: 0 a
// warp takes 32 cells at a time, 1 (the default: measured faster on every
// workload) each lane takes one cell at a time.
std::atomic<int> g_lane_queue{1};
// The automatic choice runs launches of at most this many cells on the
// warp-per-cell kernel: the thread-per-cell kernel needs about 150k cells to
// fill a B200 and is far slower below that, while the warp-per-cell kernel
// fills it with 1776 cells (12 per SM) and then stays at its throughput.
std::atomic<int> g_coop_max_cells{KPP_COOP_MAX_CELLS};

bool use_coop(const LaunchArgs& a) {
#if KPP_COOP
  if (!coop_supports(a)) return false;
  if (g_kernel_choice == 2) return true;
  if (g_kernel_choice == 1) return false;
  // A single call warm-started with per-cell Hstart (a host model's time
  // loop passing the previous call's Hexit) takes a few internal steps, and
  // the warp kernel re-stages every cell for each such call: measured on
  // B200 with saprc99 at 2^17 cells, a warm 600 s call took 203 ms there and
  // 43 ms on the thread kernel (3.3 internal steps per cell).  Those go to
  // the thread kernel; cold calls and the chained entry keep the warp kernel.
  if (a.hstart && !a.queue) return false;
  return a.ncells <= g_coop_max_cells.load();
#else
  (void)a;
  return false;
#endif
}

// Per-cell evaluation of the mechanism functions (test and tooling entry).
struct EvalArgs {
  int ncells, ld;
  const double* var;
  const double* fix;
  const double* temp;
  const double* cfactor;
  const double* sun;
  double time;
  double* rconst;
  double* vdot;
  double* jvs;
  double* scratch;
  long nslots;
};

__global__ void __launch_bounds__(128) fun_jac_kernel(const EvalArgs a) {
  const long slot = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long ld = a.ld;
  Work w(a.scratch, a.nslots, slot);
  for (long c = slot; c < a.ncells; c += a.nslots) {
    const int cell = (int)c;
    CellEnv env;
    load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, cell);
    for (int i = 0; i < NVAR; i++) w.y[i] = a.var[i * ld + cell];
    kpp_update_rconst(w.rconst, a.time, env.temp, env.cfactor, cell_sun(env, a.time), w.y,
                      env.fix);
    if (a.rconst)
      for (int i = 0; i < NREACT; i++) a.rconst[i * ld + cell] = w.rconst[i];
    if (a.vdot) {
      kpp_fun(w.y, env.fix, w.rconst, w.fcn, w.a);
      for (int i = 0; i < NVAR; i++) a.vdot[i * ld + cell] = w.fcn[i];
    }
    if (a.jvs) {
      kpp_jac_sp<false>(w.y, env.fix, w.rconst, w.jvs, w.b);
      for (int i = 0; i < LU_NZ; i++) a.jvs[i * ld + cell] = w.jvs[i];
    }
  }
}

// A batched array with a run-time leading dimension (the ABI layout).
struct StridedLd {
  double* p;
  long s;
  __device__ __forceinline__ double& operator[](int i) const { return p[(long)i * s]; }
};

__global__ void __launch_bounds__(128) decomp_solve_kernel(int ncells, int ld, double* jvs_g,
                                                           double* x_g, int* ising) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= ncells) return;
  StridedLd jvs{jvs_g + cell, ld};
  double wrow[NVAR];  // work row of the loop-form LU of large mechanisms
  ising[cell] = kpp_decomp(jvs, wrow);
  if (x_g) {
    StridedLd x{x_g + cell, ld};
    kpp_solve(jvs, x);
  }
}

// The building blocks of the discrete adjoint, one cell per thread on the
// [n][ld] arrays: J uv or J^T uv (Jac_SP_Vec / JacTR_SP_Vec) and the
// transposed LU solve (KppSolveTR).
__global__ void __launch_bounds__(128) jac_vec_kernel(int ncells, int ld, const double* jvs_g,
                                                      const double* uv_g, double* out_g,
                                                      int transposed) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= ncells) return;
  const StridedLd jvs{const_cast<double*>(jvs_g) + cell, ld};
  const StridedLd uv{const_cast<double*>(uv_g) + cell, ld};
  StridedLd out{out_g + cell, ld};
  if (transposed)
    kpp_jactr_sp_vec(jvs, uv, out);
  else
    kpp_jac_sp_vec(jvs, uv, out);
}

__global__ void __launch_bounds__(128) solve_tr_kernel(int ncells, int ld, const double* jvs_g,
                                                       const double* x_g, double* xx_g) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= ncells) return;
  const StridedLd jvs{const_cast<double*>(jvs_g) + cell, ld};
  const StridedLd x{const_cast<double*>(x_g) + cell, ld};
  StridedLd xx{xx_g + cell, ld};
  kpp_solve_tr(jvs, x, xx);
}



#if defined(KPP_SCRATCH)
constexpr bool kUsesScratch = true;
#else
constexpr bool kUsesScratch = false;
#endif

// Thread slots a launch over ncells cells uses: one per cell, at most as many
// as the device keeps resident (the rest of the cells are picked up by the
// grid-stride loop), in whole blocks.
// Blocks per SM the launches use: 0 = as many as can be resident.
std::atomic<int> g_blocks_per_sm{0};

long slots_for(int ncells) {
  static std::mutex mu;
  static std::map<int, std::pair<int, int>> resident;  // device -> (SMs, blocks per SM)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return kBlock;
  int sms, per_sm;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = resident.find(dev);
    if (it == resident.end()) {
      int n = 1, b = 1;
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
      b = occupancy_method<4>();
      if (b < 1) b = 1;
      it = resident.emplace(dev, std::make_pair(n, b)).first;
    }
    sms = it->second.first;
    per_sm = it->second.second;
  }
  const int cap = g_blocks_per_sm.load();
  if (cap > 0 && cap < per_sm) per_sm = cap;
  long res = (long)sms * per_sm * kBlock;
  long want = ((long)ncells + kBlock - 1) / kBlock * kBlock;
  return want < res ? want : res;
}

// Work storage of `nslots` thread slots with `per_slot` doubles each, in the
// warp-blocked scratch layout (whole warps).
size_t slot_bytes(long per_slot, long nslots) {
  return kUsesScratch ? (size_t)per_slot * (size_t)((nslots + kLanes - 1) / kLanes * kLanes) *
                            sizeof(double)
                      : 0;
}

size_t scratch_bytes(long nslots) { return slot_bytes(kScratchPerSlot, nslots); }

// Library-managed work buffers, one per (device, stream), grown on demand and
// kept until exit.  Growing calls cudaMalloc, which synchronises the device.
int cached_scratch(cudaStream_t stream, size_t bytes, double** out) {
  static std::mutex mu;
  static std::map<std::pair<int, cudaStream_t>, std::pair<void*, size_t>> cache;
  *out = nullptr;
  if (bytes == 0) return KPP_B200_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  std::lock_guard<std::mutex> lock(mu);
  auto& entry = cache[{dev, stream}];
  if (entry.second < bytes) {
    if (entry.first) {
      cudaStreamSynchronize(stream);
      cudaFree(entry.first);
      entry = {nullptr, 0};
    }
    void* p = nullptr;
    e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return cuda_fail("cudaMalloc(workspace)", e);
    entry = {p, bytes};
  }
  *out = (double*)entry.first;
  return KPP_B200_OK;
}

// Work-queue counter, one per (device, stream), kept until exit.
int cached_counter(cudaStream_t stream, int** out) {
  static std::mutex mu;
  static std::map<std::pair<int, cudaStream_t>, int*> cache;
  *out = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  std::lock_guard<std::mutex> lock(mu);
  int*& p = cache[{dev, stream}];
  if (!p) {
    e = cudaMalloc(&p, 256);
    if (e != cudaSuccess) {
      p = nullptr;
      return cuda_fail("cudaMalloc(queue counter)", e);
    }
  }
  *out = p;
  return KPP_B200_OK;
}

size_t scratch_capacity_doubles(const LaunchArgs& a) { return a.scratch_doubles; }

int launch_rosenbrock(LaunchArgs& a, cudaStream_t s) {
#if KPP_COOP
  if (use_coop(a)) {
    switch (a.ipar[3]) {
      case 1: return launch_method_coop<1>(a, s);
      case 2: return launch_method_coop<2>(a, s);
      case 3: return launch_method_coop<3>(a, s);
      case 5: return launch_method_coop<5>(a, s);
      default: return launch_method_coop<4>(a, s);
    }
  }
#endif
  const int grid = (int)(a.nslots / kBlock);
  // Invalid methods are reported per cell by the validation in
  // rosenbrock_cell (IERR = -2); any valid instance does that.
  switch (a.ipar[3]) {
    case 1: return launch_method<1>(a, grid, s);
    case 2: return launch_method<2>(a, grid, s);
    case 3: return launch_method<3>(a, grid, s);
    case 5: return launch_method<5>(a, grid, s);
    default: return launch_method<4>(a, grid, s);
  }
}

int fill_args(LaunchArgs& a, int ncells, int ld, double* var, const double* fix,
              const double* temp, const double* cfactor, const double* sun,
              const double* tstart, const double* tend, const double* atol, const double* rtol,
              const int* ipar, const double* rpar, const double* hstart, int* istatus,
              double* rstatus, int* ierr) {
  if (ncells < 0 || ld < ncells) return fail(KPP_B200_EINVAL, "need 0 <= ncells <= ld");
  if (ncells > 0 && (!var || !temp || !tstart || !tend || !atol || !rtol || !ipar || !rpar ||
                     !istatus || !rstatus || !ierr || (KPP_NFIX_TRUE > 0 && !fix)))
    return fail(KPP_B200_EINVAL, "null argument");
  a.ncells = ncells;
  a.ld = ld;
  a.var = var;
  a.fix = fix;
  a.temp = temp;
  a.cfactor = cfactor;
  a.sun = sun;
  a.tstart = tstart;
  a.tend = tend;
  a.atol = atol;
  a.rtol = rtol;
  a.hstart = hstart;
  a.istatus = istatus;
  a.rstatus = rstatus;
  a.ierr = ierr;
  a.scratch = nullptr;
  a.scratch_doubles = 0;
  a.nslots = 0;
  a.order = nullptr;
  a.queue = nullptr;
  a.nchain = 0;
  a.chain_dt = 0.0;
  a.lane_queue = 0;
  if (ipar) std::memcpy(a.ipar, ipar, sizeof a.ipar);
  if (rpar) std::memcpy(a.rpar, rpar, sizeof a.rpar);
  return KPP_B200_OK;
}


// ---- allocation-free variant -------------------------------------------------
// For callers that cannot allocate device memory: the work arrays of the
// allocation-free entry live in this file-scope device array, sized for
// kStaticMaxCells cells (one thread slot each, warp-blocked layout).  Every GPU
// that loads the library holds it until the process exits.  Host code must not
// use the array's name as a device address (on the host it names a host-side
// stand-in); static_scratch() obtains the device address per device.
// 1024 cells while that stays within 64 MB (saprc99: 21 MB); 128 cells for
// mechanisms with larger per-cell work arrays (MCM isoprene: 22 MB).
constexpr int kStaticMaxCells =
    (kScratchPerSlot * 8L * 1024L <= (64L << 20)) ? 1024 : 128;
static_assert(kStaticMaxCells % kBlock == 0, "whole blocks of thread slots");
#if defined(KPP_SCRATCH)
static __device__ __align__(256) double g_static_scratch[(size_t)kScratchPerSlot * kStaticMaxCells];
#endif

// Device address of g_static_scratch on the current device (nullptr for
// mechanisms whose work arrays are thread-local).  Looked up with
// cudaGetSymbolAddress on the first call per device, with that device current;
// that first call is refused while `stream` is being captured (the lookup can
// load the module, which a capture must not see).
int static_scratch(cudaStream_t stream, double** out) {
  *out = nullptr;
#if defined(KPP_SCRATCH)
  static std::mutex mu;
  static std::map<int, double*> addr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  std::lock_guard<std::mutex> lock(mu);
  auto it = addr.find(dev);
  if (it == addr.end()) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(stream, &cap);
    if (e != cudaSuccess) return cuda_fail("cudaStreamIsCapturing", e);
    if (cap != cudaStreamCaptureStatusNone)
      return fail(KPP_B200_EINVAL,
                  "kpp_b200_rosenbrock_static: the first call on a device must come before any "
                  "stream capture (call once before capture)");
    double* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_static_scratch);
    if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress(g_static_scratch)", e);
    it = addr.emplace(dev, p).first;
  }
  *out = it->second;
#endif
  return KPP_B200_OK;
}

// ---- host-buffer pipeline ---------------------------------------------------
// Device buffers of one chunk (ABI layout, leading dimension = chunk size).
struct ChunkBuffers {
  long cap = 0;
  double *var = nullptr, *fix = nullptr, *temp = nullptr, *cfactor = nullptr, *sun = nullptr;
  double *tstart = nullptr, *tend = nullptr, *hstart = nullptr, *rstatus = nullptr;
  double *atol = nullptr, *rtol = nullptr;
  int *istatus = nullptr, *ierr = nullptr;
  cudaStream_t stream = nullptr;

  void release() {
    for (void* p : {(void*)var, (void*)fix, (void*)temp, (void*)cfactor, (void*)sun,
                    (void*)tstart, (void*)tend, (void*)hstart, (void*)rstatus, (void*)atol,
                    (void*)rtol, (void*)istatus, (void*)ierr})
      if (p) cudaFree(p);
    *this = ChunkBuffers{0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                         nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, stream};
  }

  int ensure(long n) {
    if (!stream) {
      cudaError_t e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail("cudaStreamCreate", e);
    }
    if (cap >= n) return KPP_B200_OK;
    release();
    size_t d = sizeof(double);
    struct { void** p; size_t bytes; } want[] = {
        {(void**)&var, (size_t)NVAR * n * d}, {(void**)&fix, (size_t)(NFIX_TRUE > 0 ? NFIX_TRUE : 1) * n * d},
        {(void**)&temp, n * d}, {(void**)&cfactor, n * d}, {(void**)&sun, n * d},
        {(void**)&tstart, n * d}, {(void**)&tend, n * d}, {(void**)&hstart, n * d},
        {(void**)&rstatus, 3 * n * d}, {(void**)&atol, NVAR * d}, {(void**)&rtol, NVAR * d},
        {(void**)&istatus, 8 * n * sizeof(int)}, {(void**)&ierr, n * sizeof(int)}};
    for (auto& w : want) {
      cudaError_t e = cudaMalloc(w.p, w.bytes);
      if (e != cudaSuccess) {
        release();
        return cuda_fail("cudaMalloc(chunk buffers)", e);
      }
    }
    cap = n;
    return KPP_B200_OK;
  }
};

// rows x cols block of a host ABI array (leading dimension ld, first column c0)
// to/from a device array with leading dimension dld.
inline cudaError_t copy_rows(void* dst, long dld, const void* src, long sld, long c0, long cols,
                             long rows, size_t elem, cudaMemcpyKind kind, cudaStream_t s,
                             bool src_offset) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  const char* sp = (const char*)src + (src_offset ? c0 * elem : 0);
  char* dp = (char*)dst + (src_offset ? 0 : c0 * elem);
  return cudaMemcpy2DAsync(dp, dld * elem, sp, sld * elem, cols * elem, rows, kind, s);
}

// The host-array entries: chunks of cells copied in, integrated and copied
// out on two alternating streams.  `which`: 0 Rosenbrock (rstatus 2 rows), 1
// SDIRK, 2 Runge-Kutta (3 rows; no hstart).
int host_pipeline(int ncells, int ld, double* var, const double* fix, const double* temp,
                  const double* cfactor, const double* sun, const double* tstart,
                  const double* tend, const double* atol, const double* rtol, const int* ipar,
                  const double* rpar, const double* hstart, int* istatus, double* rstatus,
                  int* ierr, int chunk, int which) {
  static std::mutex mu;
  static std::map<int, ChunkBuffers[2]> per_device;
  std::lock_guard<std::mutex> lock(mu);  // one host pipeline per process at a time
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  long csz = chunk > 0 ? chunk : (1L << 18);
  if (csz > ncells) csz = ncells;
  ChunkBuffers* bufs = per_device[dev];
  const int ntol = (ipar[1] == 0) ? NVAR : 1;
  for (int b = 0; b < 2; b++) {
    int rc = bufs[b].ensure(csz);
    if (rc != KPP_B200_OK) return rc;
    e = cudaMemcpyAsync(bufs[b].atol, atol, ntol * sizeof(double), cudaMemcpyHostToDevice,
                        bufs[b].stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(bufs[b].rtol, rtol, ntol * sizeof(double), cudaMemcpyHostToDevice,
                          bufs[b].stream);
    if (e != cudaSuccess) return cuda_fail("tolerance copy", e);
  }
  const auto H2D = cudaMemcpyHostToDevice;
  const auto D2H = cudaMemcpyDeviceToHost;
  long nchunks = ((long)ncells + csz - 1) / csz;
  for (long c = 0; c < nchunks; c++) {
    ChunkBuffers& B = bufs[c & 1];
    cudaStream_t s = B.stream;
    long c0 = c * csz, n = ((long)ncells - c0 < csz) ? (long)ncells - c0 : csz;
    e = copy_rows(B.var, csz, var, ld, c0, n, NVAR, sizeof(double), H2D, s, true);
    if (e == cudaSuccess && NFIX_TRUE > 0)
      e = copy_rows(B.fix, csz, fix, ld, c0, n, NFIX_TRUE, sizeof(double), H2D, s, true);
    if (e == cudaSuccess) e = copy_rows(B.temp, csz, temp, ld, c0, n, 1, sizeof(double), H2D, s, true);
    if (e == cudaSuccess && cfactor)
      e = copy_rows(B.cfactor, csz, cfactor, ld, c0, n, 1, sizeof(double), H2D, s, true);
    if (e == cudaSuccess && sun) e = copy_rows(B.sun, csz, sun, ld, c0, n, 1, sizeof(double), H2D, s, true);
    if (e == cudaSuccess) e = copy_rows(B.tstart, csz, tstart, ld, c0, n, 1, sizeof(double), H2D, s, true);
    if (e == cudaSuccess) e = copy_rows(B.tend, csz, tend, ld, c0, n, 1, sizeof(double), H2D, s, true);
    if (e == cudaSuccess && hstart)
      e = copy_rows(B.hstart, csz, hstart, ld, c0, n, 1, sizeof(double), H2D, s, true);
    if (e != cudaSuccess) return cuda_fail("host->device copy", e);

    LaunchArgs a;
    fill_args(a, (int)n, (int)csz, B.var, B.fix, B.temp, cfactor ? B.cfactor : nullptr,
              sun ? B.sun : nullptr, B.tstart, B.tend, B.atol, B.rtol, ipar, rpar,
              hstart ? B.hstart : nullptr, B.istatus, B.rstatus, B.ierr);
    a.nslots = slots_for((int)n);
    int rc;
    if (which == 0) {
      if (!use_coop(a)) {  // the warp-per-cell kernel needs no work buffer
        rc = cached_scratch(s, scratch_bytes(a.nslots), &a.scratch);
        if (rc != KPP_B200_OK) return rc;
        a.scratch_doubles = scratch_bytes(a.nslots) / sizeof(double);
      }
      rc = launch_rosenbrock(a, s);
    } else {
      const long per = which == 1 ? kSdirkPerSlot : kRkPerSlot;
      const size_t bytes = slot_bytes(per, a.nslots);
      rc = cached_scratch(s, bytes, &a.scratch);
      if (rc != KPP_B200_OK) return rc;
      a.scratch_doubles = bytes / sizeof(double);
      rc = which == 1 ? launch_sdirk(a, (int)(a.nslots / kBlock), s)
                      : launch_rk(a, (int)(a.nslots / kBlock), s);
    }
    if (rc != KPP_B200_OK) return rc;

    const long rst_rows = which == 0 ? 2 : 3;
    e = copy_rows(var, ld, B.var, csz, c0, n, NVAR, sizeof(double), D2H, s, false);
    if (e == cudaSuccess) e = copy_rows(istatus, ld, B.istatus, csz, c0, n, 8, sizeof(int), D2H, s, false);
    if (e == cudaSuccess) e = copy_rows(rstatus, ld, B.rstatus, csz, c0, n, rst_rows, sizeof(double), D2H, s, false);
    if (e == cudaSuccess) e = copy_rows(ierr, ld, B.ierr, csz, c0, n, 1, sizeof(int), D2H, s, false);
    if (e != cudaSuccess) return cuda_fail("device->host copy", e);
  }
  for (int b = 0; b < 2; b++) {
    e = cudaStreamSynchronize(bufs[b].stream);
    if (e != cudaSuccess) return cuda_fail("cudaStreamSynchronize", e);
  }
  return KPP_B200_OK;
}

#endif  // KPP_PART

}  // namespace kpp_b200_impl

#if KPP_PART == 0
#ifdef KPP_HOST_HEADER
#include KPP_HOST_HEADER
#else
#define KPP_NUSER 0
namespace kpp_host {
static const int kUserToKpp[1] = {-1};
}
#endif

namespace kpp_b200_impl {
// Species map of the shuffle entries on the device (user index -> KPP index,
// -1 for user species that take no part in the mechanism).
__constant__ int c_user_to_kpp[KPP_NUSER > 0 ? KPP_NUSER : 1];

// dir 0: var[kpp[k]][c] = user[k][c]; dir 1: user[k][c] = var[kpp[k]][c].
// One thread per (cell, user species), cells fastest: both sides coalesced.
__global__ void shuffle_kernel(int ncells, int nuser, int dir, double* user, long ld_user,
                               double* var, long ld) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long c = i % ncells, k = i / ncells;
  if (k >= nuser) return;
  const int f = c_user_to_kpp[k];
  if (f < 0) return;
  if (dir == 0)
    var[(long)f * ld + c] = user[k * ld_user + c];
  else
    user[k * ld_user + c] = var[(long)f * ld + c];
}

int shuffle(int ncells, double* user, long ld_user, double* var, long ld, int dir,
            cudaStream_t s) {
  if (ncells < 0 || ld < ncells || ld_user < ncells) return fail(KPP_B200_EINVAL, "bad sizes");
  if (ncells == 0 || KPP_NUSER == 0) return KPP_B200_OK;
  if (!user || !var) return fail(KPP_B200_EINVAL, "null argument");
  static int uploaded_dev = -1;  // the map is uploaded once per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  if (uploaded_dev != dev) {
    e = cudaMemcpyToSymbol(c_user_to_kpp, kpp_host::kUserToKpp, sizeof(int) * KPP_NUSER);
    if (e != cudaSuccess) return cuda_fail("cudaMemcpyToSymbol(species map)", e);
    uploaded_dev = dev;
  }
  const long total = (long)ncells * KPP_NUSER;
  shuffle_kernel<<<(int)((total + 255) / 256), 256, 0, s>>>(ncells, KPP_NUSER, dir, user,
                                                              ld_user, var, ld);
  return check_launch("shuffle_kernel");
}
}  // namespace kpp_b200_impl

using namespace kpp_b200_impl;

extern "C" {

int kpp_b200_user_species(int* nuser, int* kpp_index) {
  if (nuser) *nuser = KPP_NUSER;
  if (kpp_index)
    for (int k = 0; k < KPP_NUSER; k++) kpp_index[k] = kpp_host::kUserToKpp[k];
  return KPP_B200_OK;
}

int kpp_b200_shuffle_user2kpp(int ncells, int ld_user, const double* v_user, int ld,
                              double* var, void* stream) {
  return shuffle(ncells, const_cast<double*>(v_user), ld_user, var, ld, 0, (cudaStream_t)stream);
}

int kpp_b200_shuffle_kpp2user(int ncells, int ld, const double* var, int ld_user,
                              double* v_user, void* stream) {
  return shuffle(ncells, v_user, ld_user, const_cast<double*>(var), ld, 1, (cudaStream_t)stream);
}


int kpp_b200_dims(int* dims) {
  if (!dims) return fail(KPP_B200_EINVAL, "dims is NULL");
  dims[0] = KPP_NVAR;
  dims[1] = KPP_NFIX_TRUE;
  dims[2] = KPP_NSPEC;
  dims[3] = KPP_NREACT;
  dims[4] = KPP_LU_NONZERO;
  dims[5] = KPP_NONZERO;
  return KPP_B200_OK;
}

const char* kpp_b200_mechanism_name(void) { return KPP_MECH_NAME; }

const char* kpp_b200_species_name(int i) {
  return (i >= 0 && i < KPP_NSPEC) ? kpp_mech::kSpeciesNames[i] : "";
}

int kpp_b200_initial_values(double* c, double* cfactor) {
  if (!c || !cfactor) return fail(KPP_B200_EINVAL, "null argument");
  for (int i = 0; i < KPP_NSPEC; i++) c[i] = kpp_mech::kInitialValues[i] * KPP_CFACTOR;
  *cfactor = KPP_CFACTOR;
  return KPP_B200_OK;
}

int kpp_b200_lu_pattern(int* irow, int* icol, int* crow, int* diag) {
  if (!irow || !icol || !crow || !diag) return fail(KPP_B200_EINVAL, "null argument");
  for (int i = 0; i < KPP_LU_NONZERO; i++) {
    irow[i] = kpp_mech::kLuIRow[i];
    icol[i] = kpp_mech::kLuICol[i];
  }
  for (int i = 0; i <= KPP_NVAR; i++) {
    crow[i] = kpp_mech::kLuCRow[i];
    diag[i] = kpp_mech::kLuDiag[i];
  }
  return KPP_B200_OK;
}

int kpp_b200_rosenbrock(int ncells, int ld, double* var, const double* fix, const double* temp,
                        const double* cfactor, const double* sun, const double* tstart,
                        const double* tend, const double* atol, const double* rtol,
                        const int* ipar, const double* rpar, const double* hstart,
                        int* istatus, double* rstatus, int* ierr, void* stream) {
  LaunchArgs a;
  int rc = fill_args(a, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol, ipar,
                     rpar, hstart, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (!use_coop(a)) {  // the warp-per-cell kernel needs no work buffer
    a.nslots = slots_for(ncells);
    rc = cached_scratch(s, scratch_bytes(a.nslots), &a.scratch);
    if (rc != KPP_B200_OK) return rc;
    a.scratch_doubles = scratch_bytes(a.nslots) / sizeof(double);
  }
  return launch_rosenbrock(a, s);
}

int kpp_b200_sdirk(int ncells, int ld, double* var, const double* fix, const double* temp,
                   const double* cfactor, const double* sun, const double* tstart,
                   const double* tend, const double* atol, const double* rtol,
                   const int* icntrl, const double* rcntrl, int* istatus, double* rstatus,
                   int* ierr, void* stream) {
  LaunchArgs a;
  int rc = fill_args(a, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol,
                     icntrl, rcntrl, nullptr, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  a.nslots = slots_for(ncells);
  const size_t bytes = slot_bytes(kSdirkPerSlot, a.nslots);
  rc = cached_scratch(s, bytes, &a.scratch);
  if (rc != KPP_B200_OK) return rc;
  a.scratch_doubles = bytes / sizeof(double);
  return launch_sdirk(a, (int)(a.nslots / kBlock), s);
}

int kpp_b200_runge_kutta(int ncells, int ld, double* var, const double* fix,
                         const double* temp, const double* cfactor, const double* sun,
                         const double* tstart, const double* tend, const double* atol,
                         const double* rtol, const int* icntrl, const double* rcntrl,
                         int* istatus, double* rstatus, int* ierr, void* stream) {
  LaunchArgs a;
  int rc = fill_args(a, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol,
                     icntrl, rcntrl, nullptr, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  a.nslots = slots_for(ncells);
  const size_t bytes = slot_bytes(kRkPerSlot, a.nslots);
  rc = cached_scratch(s, bytes, &a.scratch);
  if (rc != KPP_B200_OK) return rc;
  a.scratch_doubles = bytes / sizeof(double);
  return launch_rk(a, (int)(a.nslots / kBlock), s);
}

size_t kpp_b200_rosenbrock_adj_work_bytes(int ld, int nadj, int bufsize, int save_lu) {
#if defined(KPP_NHESS)
  if (ld < 0 || nadj < 0 || bufsize < 1) return 0;
  return (size_t)kpp_adj::adj_layout(nadj, bufsize, save_lu != 0).total * (size_t)ld *
         sizeof(double);
#else
  (void)ld; (void)nadj; (void)bufsize; (void)save_lu;
  return 0;
#endif
}

int kpp_b200_rosenbrock_adj(int ncells, int ld, double* var, const double* fix,
                            const double* temp, const double* cfactor, const double* sun,
                            const double* tstart, const double* tend, const double* atol,
                            const double* rtol, int nadj, double* lambda, const int* icntrl,
                            const double* rcntrl, int bufsize, double* work, size_t work_bytes,
                            int* istatus, double* rstatus, int* ierr, void* stream) {
#if defined(KPP_NHESS)
  LaunchArgs a;
  int rc = fill_args(a, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol,
                     icntrl, rcntrl, nullptr, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK) return rc;
  if (nadj < 0) return fail(KPP_B200_EINVAL, "nadj must be >= 0");
  if (bufsize < 1) return fail(KPP_B200_EINVAL, "bufsize must be >= 1");
  if (ncells == 0) return KPP_B200_OK;
  if (nadj > 0 && !lambda) return fail(KPP_B200_EINVAL, "null lambda");
  if (icntrl[6] == 3 || icntrl[6] == 4)
    return fail(KPP_B200_EINVAL, "ICNTRL[6] 3 and 4 (continuous adjoints) are not built");
  const size_t need = kpp_b200_rosenbrock_adj_work_bytes(ld, nadj, bufsize, icntrl[7]);
  if (!work || work_bytes < need) return fail(KPP_B200_EINVAL, "work buffer too small");
  return launch_adj(a, lambda, nadj, bufsize, work, (cudaStream_t)stream);
#else
  (void)ncells; (void)ld; (void)var; (void)fix; (void)temp; (void)cfactor; (void)sun;
  (void)tstart; (void)tend; (void)atol; (void)rtol; (void)nadj; (void)lambda; (void)icntrl;
  (void)rcntrl; (void)bufsize; (void)work; (void)work_bytes; (void)istatus; (void)rstatus;
  (void)ierr; (void)stream;
  return fail(KPP_B200_EINVAL,
              "this library has no Hessian: the adjoint is in the library built on KPP's own "
              "generator (libkpp_b200_<mech>_kpproute.so)");
#endif
}

int kpp_b200_rosenbrock_chain(int ncells, int ld, double* var, const double* fix,
                              const double* temp, const double* cfactor, const double* sun,
                              const double* tstart, double dt, int ncalls, const double* atol,
                              const double* rtol, const int* ipar, const double* rpar,
                              const double* hstart, const int* order, int* istatus,
                              double* rstatus, int* ierr, void* stream) {
  LaunchArgs a;
  // tend is not read in chained mode; tstart stands in for the null check
  int rc = fill_args(a, ncells, ld, var, fix, temp, cfactor, sun, tstart, tstart, atol, rtol,
                     ipar, rpar, hstart, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK) return rc;
  if (ncalls < 1) return fail(KPP_B200_EINVAL, "ncalls must be >= 1");
  if (ncells == 0) return KPP_B200_OK;
  cudaStream_t s = (cudaStream_t)stream;
  a.nchain = ncalls;
  a.chain_dt = dt;
  a.order = order;
  a.lane_queue = g_lane_queue.load();
  if (!use_coop(a)) {  // the warp-per-cell kernel needs no work buffer
    a.nslots = slots_for(ncells);
    rc = cached_scratch(s, scratch_bytes(a.nslots), &a.scratch);
    if (rc != KPP_B200_OK) return rc;
    a.scratch_doubles = scratch_bytes(a.nslots) / sizeof(double);
  }
  rc = cached_counter(s, &a.queue);
  if (rc != KPP_B200_OK) return rc;
  cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(int), s);
  if (e != cudaSuccess) return cuda_fail("cudaMemsetAsync(queue counter)", e);
  return launch_rosenbrock(a, s);
}

size_t kpp_b200_workspace_bytes(int ncells) {
  return ncells > 0 ? scratch_bytes(slots_for(ncells)) : 0;
}

int kpp_b200_rosenbrock_ws(int ncells, int ld, double* var, const double* fix, const double* temp,
                           const double* cfactor, const double* sun, const double* tstart,
                           const double* tend, const double* atol, const double* rtol,
                           const int* ipar, const double* rpar, const double* hstart,
                           int* istatus, double* rstatus, int* ierr, void* workspace,
                           size_t workspace_bytes, void* stream) {
  LaunchArgs a;
  int rc = fill_args(a, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol, ipar,
                     rpar, hstart, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  a.nslots = slots_for(ncells);
  if (kUsesScratch && !use_coop(a)) {
    if (!workspace || workspace_bytes < scratch_bytes(a.nslots))
      return fail(KPP_B200_EINVAL, "workspace smaller than kpp_b200_workspace_bytes()");
    a.scratch = (double*)workspace;
    a.scratch_doubles = workspace_bytes / sizeof(double);
  }
  return launch_rosenbrock(a, (cudaStream_t)stream);
}

int kpp_b200_rosenbrock_static(int ncells, int ld, double* var, const double* fix,
                               const double* temp, const double* cfactor, const double* sun,
                               const double* tstart, const double* tend, const double* atol,
                               const double* rtol, const int* ipar, const double* rpar,
                               const double* hstart, int* istatus, double* rstatus, int* ierr,
                               void* stream) {
  LaunchArgs a;
  int rc = fill_args(a, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol, ipar,
                     rpar, hstart, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  if (ncells > kStaticMaxCells) {
    std::snprintf(g_last_error, sizeof g_last_error,
                  "kpp_b200_rosenbrock_static: %d cells exceed its maximum of %d cells per call",
                  ncells, kStaticMaxCells);
    return KPP_B200_EINVAL;
  }
  // one thread slot per cell, in whole blocks: at most kStaticMaxCells slots
  a.nslots = ((long)ncells + kBlock - 1) / kBlock * kBlock;
  rc = static_scratch((cudaStream_t)stream, &a.scratch);
  if (rc != KPP_B200_OK) return rc;
  a.scratch_doubles = a.scratch ? (size_t)kScratchPerSlot * kStaticMaxCells : 0;
  return launch_rosenbrock(a, (cudaStream_t)stream);
}

int kpp_b200_rosenbrock_host(int ncells, int ld, double* var, const double* fix,
                             const double* temp, const double* cfactor, const double* sun,
                             const double* tstart, const double* tend, const double* atol,
                             const double* rtol, const int* ipar, const double* rpar,
                             const double* hstart, int* istatus, double* rstatus, int* ierr,
                             int chunk) {
  LaunchArgs chk;
  int rc = fill_args(chk, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol,
                     ipar, rpar, hstart, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  return host_pipeline(ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol, ipar,
                       rpar, hstart, istatus, rstatus, ierr, chunk, 0);
}

int kpp_b200_sdirk_host(int ncells, int ld, double* var, const double* fix, const double* temp,
                        const double* cfactor, const double* sun, const double* tstart,
                        const double* tend, const double* atol, const double* rtol,
                        const int* icntrl, const double* rcntrl, int* istatus, double* rstatus,
                        int* ierr, int chunk) {
  LaunchArgs chk;
  int rc = fill_args(chk, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol,
                     icntrl, rcntrl, nullptr, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  return host_pipeline(ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol, icntrl,
                       rcntrl, nullptr, istatus, rstatus, ierr, chunk, 1);
}

int kpp_b200_runge_kutta_host(int ncells, int ld, double* var, const double* fix,
                              const double* temp, const double* cfactor, const double* sun,
                              const double* tstart, const double* tend, const double* atol,
                              const double* rtol, const int* icntrl, const double* rcntrl,
                              int* istatus, double* rstatus, int* ierr, int chunk) {
  LaunchArgs chk;
  int rc = fill_args(chk, ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol,
                     icntrl, rcntrl, nullptr, istatus, rstatus, ierr);
  if (rc != KPP_B200_OK || ncells == 0) return rc;
  return host_pipeline(ncells, ld, var, fix, temp, cfactor, sun, tstart, tend, atol, rtol, icntrl,
                       rcntrl, nullptr, istatus, rstatus, ierr, chunk, 2);
}

int kpp_b200_fun_jac(int ncells, int ld, const double* var, const double* fix,
                     const double* temp, const double* cfactor, const double* sun, double time,
                     double* rconst, double* vdot, double* jvs, void* stream) {
  if (ncells < 0 || ld < ncells) return fail(KPP_B200_EINVAL, "need 0 <= ncells <= ld");
  if (ncells == 0) return KPP_B200_OK;
  if (!var || !temp || (KPP_NFIX_TRUE > 0 && !fix)) return fail(KPP_B200_EINVAL, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  EvalArgs a{ncells, ld, var, fix, temp, cfactor, sun, time, rconst, vdot, jvs, nullptr, 0};
  a.nslots = slots_for(ncells);
  int rc = cached_scratch(s, scratch_bytes(a.nslots), &a.scratch);
  if (rc != KPP_B200_OK) return rc;
  fun_jac_kernel<<<(int)(a.nslots / kBlock), kBlock, 0, s>>>(a);
  return check_launch("fun_jac_kernel");
}

int kpp_b200_decomp_solve(int ncells, int ld, double* jvs, double* x, int* ising, void* stream) {
  if (ncells < 0 || ld < ncells) return fail(KPP_B200_EINVAL, "need 0 <= ncells <= ld");
  if (ncells == 0) return KPP_B200_OK;
  if (!jvs || !ising) return fail(KPP_B200_EINVAL, "null argument");
  decomp_solve_kernel<<<(ncells + kBlock - 1) / kBlock, kBlock, 0, (cudaStream_t)stream>>>(
      ncells, ld, jvs, x, ising);
  return check_launch("decomp_solve_kernel");
}

int kpp_b200_jac_vec(int ncells, int ld, const double* jvs, const double* uv, double* out,
                     int transposed, void* stream) {
  if (ncells < 0 || ld < ncells) return fail(KPP_B200_EINVAL, "need 0 <= ncells <= ld");
  if (ncells == 0) return KPP_B200_OK;
  if (!jvs || !uv || !out) return fail(KPP_B200_EINVAL, "null argument");
  if (uv == out) return fail(KPP_B200_EINVAL, "out must not be uv");
  jac_vec_kernel<<<(ncells + kBlock - 1) / kBlock, kBlock, 0, (cudaStream_t)stream>>>(
      ncells, ld, jvs, uv, out, transposed);
  return check_launch("jac_vec_kernel");
}

int kpp_b200_solve_tr(int ncells, int ld, const double* jvs, const double* x, double* xx,
                      void* stream) {
  if (ncells < 0 || ld < ncells) return fail(KPP_B200_EINVAL, "need 0 <= ncells <= ld");
  if (ncells == 0) return KPP_B200_OK;
  if (!jvs || !x || !xx) return fail(KPP_B200_EINVAL, "null argument");
  solve_tr_kernel<<<(ncells + kBlock - 1) / kBlock, kBlock, 0, (cudaStream_t)stream>>>(
      ncells, ld, jvs, x, xx);
  return check_launch("solve_tr_kernel");
}

const char* kpp_b200_last_error(void) { return g_last_error; }

int kpp_b200_set_kernel(int which) {
  if (which < 0 || which > 2) return fail(KPP_B200_EINVAL, "kernel choice must be 0, 1 or 2");
  g_kernel_choice = which;
  return KPP_B200_OK;
}

int kpp_b200_get_kernel(void) {
#if KPP_COOP
  return g_kernel_choice == 2 ? 2 : 1;
#else
  return 1;
#endif
}

int kpp_b200_set_queue_lanes(int per_lane) {
  if (per_lane < 0 || per_lane > 1) return fail(KPP_B200_EINVAL, "queue granularity must be 0 or 1");
  g_lane_queue.store(per_lane);
  return KPP_B200_OK;
}

int kpp_b200_get_queue_lanes(void) { return g_lane_queue.load(); }

int kpp_b200_set_auto_warp_cells(int ncells) {
  if (ncells < 0) return fail(KPP_B200_EINVAL, "the cell limit must be >= 0");
  g_coop_max_cells.store(ncells);
  return KPP_B200_OK;
}

int kpp_b200_get_auto_warp_cells(void) { return g_coop_max_cells.load(); }

int kpp_b200_set_blocks_per_sm(int blocks) {
  if (blocks < 0 || blocks > 64) return fail(KPP_B200_EINVAL, "blocks per SM must be 0..64");
  g_blocks_per_sm.store(blocks);
  return KPP_B200_OK;
}

int kpp_b200_get_blocks_per_sm(void) { return g_blocks_per_sm.load(); }

}  // extern "C"

#endif  // KPP_PART == 0
