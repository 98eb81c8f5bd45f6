// Per-cell definitions shared by the integrators of kpp_rosenbrock.cu and by
// host builds of them (test infrastructure): mechanism sizes, the macros of
// int/rosenbrock.c:1-3, the Rosenbrock tableaux, launch arguments, work
// layouts, the cell environment, the hoisting of rate constants and the
// vector operations of util/blas.c.
// Included inside namespace kpp_b200_impl, after the mechanism header.
#pragma once

constexpr int NVAR = KPP_NVAR;
constexpr int NFIX = KPP_NFIX;
constexpr int NFIX_TRUE = KPP_NFIX_TRUE;
constexpr int NREACT = KPP_NREACT;
constexpr int LU_NZ = KPP_LU_NONZERO;

// Unit roundoff of WLAMCH('E') (util/blas.c:150-183): 2^-52.
constexpr double kRoundoff = 2.220446049250313080847e-16;
constexpr double kDeltaMin = 1.0e-6;  // int/rosenbrock.c:11

// int/rosenbrock.c:1-3 as functions; ABS keeps the macro's unparenthesised
// negation: ABS(a - b) of a negative difference evaluates -a - b.
__device__ __forceinline__ double ros_max(double a, double b) { return (a >= b) ? a : b; }
__device__ __forceinline__ double ros_min(double b, double c) { return (b < c) ? b : c; }
__device__ __forceinline__ double ros_abs(double x) { return (x >= 0) ? x : -x; }
__device__ __forceinline__ double ros_abs_diff(double a, double b) {
  return ((a - b) >= 0) ? (a - b) : (-a - b);
}

// Rosenbrock method coefficients (int/rosenbrock.c:779-1222).  A and C are
// strictly lower triangular, stored row-wise: A(i,j) = A[(i-1)(i-2)/2 + j-1].
struct Tableau {
  int S;
  double A[15], C[15], M[6], E[6], Alpha[6], Gamma[6], ELO;
  bool NewF[6];
};

__host__ __device__ constexpr Tableau make_tableau(int method) {
  Tableau t{};
  if (method == 1) {  // Ros2
    const double g = 1.70710678118655;
    t.S = 2;
    t.A[0] = 1.0 / g;
    t.C[0] = (-2.0) / g;
    t.NewF[0] = true; t.NewF[1] = true;
    t.M[0] = (3.0) / (2.0 * g); t.M[1] = (1.0) / (2.0 * g);
    t.E[0] = 1.0 / (2.0 * g); t.E[1] = 1.0 / (2.0 * g);
    t.ELO = 2.0;
    t.Alpha[0] = 0.0; t.Alpha[1] = 1.0;
    t.Gamma[0] = g; t.Gamma[1] = -g;
  } else if (method == 2) {  // Ros3
    t.S = 3;
    t.A[0] = 1.0; t.A[1] = 1.0; t.A[2] = 0.0;
    t.C[0] = -1.0156171083877702091975600115545;
    t.C[1] = 4.0759956452537699824805835358067;
    t.C[2] = 9.2076794298330791242156818474003;
    t.NewF[0] = true; t.NewF[1] = true; t.NewF[2] = false;
    t.M[0] = 1.0;
    t.M[1] = 6.1697947043828245592553615689730;
    t.M[2] = -0.4277225654321857332623837380651;
    t.E[0] = 0.5;
    t.E[1] = -2.9079558716805469821718236208017;
    t.E[2] = 0.2235406989781156962736090927619;
    t.ELO = 3.0;
    t.Alpha[0] = 0.0;
    t.Alpha[1] = 0.43586652150845899941601945119356;
    t.Alpha[2] = 0.43586652150845899941601945119356;
    t.Gamma[0] = 0.43586652150845899941601945119356;
    t.Gamma[1] = 0.24291996454816804366592249683314;
    t.Gamma[2] = 2.1851380027664058511513169485832;
  } else if (method == 3) {  // Ros4
    t.S = 4;
    t.A[0] = 0.2000000000000000e+01;
    t.A[1] = 0.1867943637803922e+01;
    t.A[2] = 0.2344449711399156;
    t.A[3] = t.A[1]; t.A[4] = t.A[2]; t.A[5] = 0.0;
    t.C[0] = -0.7137615036412310e+01;
    t.C[1] = 0.2580708087951457e+01;
    t.C[2] = 0.6515950076447975;
    t.C[3] = -0.2137148994382534e+01;
    t.C[4] = -0.3214669691237626;
    t.C[5] = -0.6949742501781779;
    t.NewF[0] = true; t.NewF[1] = true; t.NewF[2] = true; t.NewF[3] = false;
    t.M[0] = 0.2255570073418735e+01;
    t.M[1] = 0.2870493262186792;
    t.M[2] = 0.4353179431840180;
    t.M[3] = 0.1093502252409163e+01;
    t.E[0] = -0.2815431932141155;
    t.E[1] = -0.7276199124938920e-01;
    t.E[2] = -0.1082196201495311;
    t.E[3] = -0.1093502252409163e+01;
    t.ELO = 4.0;
    t.Alpha[0] = 0.0;
    t.Alpha[1] = 0.1145640000000000e+01;
    t.Alpha[2] = 0.6552168638155900;
    t.Alpha[3] = t.Alpha[2];
    t.Gamma[0] = 0.5728200000000000;
    t.Gamma[1] = -0.1769193891319233e+01;
    t.Gamma[2] = 0.7592633437920482;
    t.Gamma[3] = -0.1049021087100450;
  } else if (method == 4) {  // Rodas3
    t.S = 4;
    t.A[0] = 0.0; t.A[1] = 2.0; t.A[2] = 0.0; t.A[3] = 2.0; t.A[4] = 0.0; t.A[5] = 1.0;
    t.C[0] = 4.0; t.C[1] = 1.0; t.C[2] = -1.0; t.C[3] = 1.0; t.C[4] = -1.0;
    t.C[5] = -2.66666666666667;
    t.NewF[0] = true; t.NewF[1] = false; t.NewF[2] = true; t.NewF[3] = true;
    t.M[0] = 2.0; t.M[1] = 0.0; t.M[2] = 1.0; t.M[3] = 1.0;
    t.E[0] = 0.0; t.E[1] = 0.0; t.E[2] = 0.0; t.E[3] = 1.0;
    t.ELO = 3.0;
    t.Alpha[0] = 0.0; t.Alpha[1] = 0.0; t.Alpha[2] = 1.0; t.Alpha[3] = 1.0;
    t.Gamma[0] = 0.5; t.Gamma[1] = 1.5; t.Gamma[2] = 0.0; t.Gamma[3] = 0.0;
  } else if (method == 5) {  // Rodas4
    t.S = 6;
    t.Alpha[0] = 0.000; t.Alpha[1] = 0.386; t.Alpha[2] = 0.210;
    t.Alpha[3] = 0.630; t.Alpha[4] = 1.000; t.Alpha[5] = 1.000;
    t.Gamma[0] = 0.2500000000000000; t.Gamma[1] = -0.1043000000000000;
    t.Gamma[2] = 0.1035000000000000; t.Gamma[3] = -0.3620000000000023e-01;
    t.Gamma[4] = 0.0; t.Gamma[5] = 0.0;
    t.A[0] = 0.1544000000000000e+01; t.A[1] = 0.9466785280815826;
    t.A[2] = 0.2557011698983284; t.A[3] = 0.3314825187068521e+01;
    t.A[4] = 0.2896124015972201e+01; t.A[5] = 0.9986419139977817;
    t.A[6] = 0.1221224509226641e+01; t.A[7] = 0.6019134481288629e+01;
    t.A[8] = 0.1253708332932087e+02; t.A[9] = -0.6878860361058950;
    t.A[10] = t.A[6]; t.A[11] = t.A[7]; t.A[12] = t.A[8]; t.A[13] = t.A[9];
    t.A[14] = 1.0;
    t.C[0] = -0.5668800000000000e+01; t.C[1] = -0.2430093356833875e+01;
    t.C[2] = -0.2063599157091915; t.C[3] = -0.1073529058151375;
    t.C[4] = -0.9594562251023355e+01; t.C[5] = -0.2047028614809616e+02;
    t.C[6] = 0.7496443313967647e+01; t.C[7] = -0.1024680431464352e+02;
    t.C[8] = -0.3399990352819905e+02; t.C[9] = 0.1170890893206160e+02;
    t.C[10] = 0.8083246795921522e+01; t.C[11] = -0.7981132988064893e+01;
    t.C[12] = -0.3152159432874371e+02; t.C[13] = 0.1631930543123136e+02;
    t.C[14] = -0.6058818238834054e+01;
    t.M[0] = t.A[6]; t.M[1] = t.A[7]; t.M[2] = t.A[8]; t.M[3] = t.A[9];
    t.M[4] = 1.0; t.M[5] = 1.0;
    t.E[5] = 1.0;
    for (int i = 0; i < 6; i++) t.NewF[i] = true;
    t.ELO = 4.0;
  }
  return t;
}

// Everything one launch needs.  Passed by value (kernel parameter space).
struct LaunchArgs {
  int ncells, ld;
  double* var;
  const double* fix;
  const double* temp;
  const double* cfactor;
  const double* sun;
  const double* tstart;
  const double* tend;
  const double* atol;
  const double* rtol;
  const double* hstart;
  int* istatus;
  double* rstatus;
  int* ierr;
  double* scratch;  // work arrays of every thread slot (scratch layout), or null
  long nslots;      // thread slots of the grid = stride of the scratch arrays
  size_t scratch_doubles;  // capacity of `scratch`
  int ipar[20];
  double rpar[20];
  // Work queue and chained calls (kpp_b200_rosenbrock_chain); zero/null for
  // the single-call entries.
  const int* order;  // queue position -> cell, or null for the identity
  int* queue;        // device counter of cells handed out (zero at launch), or
                     // null for the grid-stride loop
  int nchain;        // > 0: that many calls [T, T + chain_dt], T += chain_dt
  double chain_dt;
  int lane_queue;    // with `queue`: each lane takes one cell at a time
};

// Whether the warp-per-cell kernel (kpp_coop.cuh) can integrate a launch: the
// mechanism has its tables and every rate constant is fixed for the call.
inline bool coop_supports(const LaunchArgs& a) {
  return KPP_COOP && KPP_RATES_DYNAMIC == 0 && (KPP_RATES_SUN == 0 || a.sun != nullptr);
}

struct Stats {
  int nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng;
};

// Scratch layout, blocked by warp: the 32 thread slots of a warp own one
// contiguous block, and element i of a per-cell work array of lane l sits at
// block[(offset_of_array + i) * 32 + l].  A warp touching the same element of
// its 32 cells issues one coalesced 256-byte access; every access is the
// lane's block pointer plus a compile-time constant below 1 MB, so it fits
// the load/store immediate offset, and the compiler can prove that different
// elements do not alias and keep, reorder and batch its loads.  The layout
// spans the launch's thread slots in whole warps (scratch_bytes).
constexpr int kLanes = 32;

struct Strided {
  double* p;
  __device__ __forceinline__ double& operator[](int i) const { return p[i * kLanes]; }
};

// Doubles of work storage one thread slot needs in the scratch layout.
constexpr int kMaxStages = 6;
constexpr long kScratchPerSlot = (long)LU_NZ + (long)kMaxStages * NVAR + 6L * NVAR +
                                 2L * NREACT + KPP_NJAC_TMP;
// ... and the SDIRK integrator (kpp_sdirk.cuh): the Jacobian kept between
// steps and the factorised matrix, five stage vectors and five vectors.
constexpr int kSdirkStages = 5;
constexpr long kSdirkPerSlot = 2L * LU_NZ + (long)(kSdirkStages + 5) * NVAR + 2L * NREACT +
                               KPP_NJAC_TMP;

#if defined(KPP_SCRATCH)
// Large mechanisms: every per-cell work array lives in the scratch buffer.
struct Work {
  Strided y, ynew, fcn0, fcn, dfdt, yerr, jvs, rconst, a, b;
  Strided k[kMaxStages];
  __device__ __forceinline__ Work(double* base, long, long slot) {
    double* block = base + (slot / kLanes) * kScratchPerSlot * kLanes + (slot % kLanes);
    long off = 0;
    auto take = [&](long n) {
      Strided v{block + off * kLanes};
      off += n;
      return v;
    };
    y = take(NVAR); ynew = take(NVAR); fcn0 = take(NVAR); fcn = take(NVAR);
    dfdt = take(NVAR); yerr = take(NVAR); jvs = take(LU_NZ);
    rconst = take(NREACT); a = take(NREACT); b = take(KPP_NJAC_TMP);
    for (int s = 0; s < kMaxStages; s++) k[s] = take(NVAR);
  }
};
#else
// Small mechanisms: work arrays are thread-local (registers).
struct Work {
  double y[NVAR], ynew[NVAR], fcn0[NVAR], fcn[NVAR], dfdt[NVAR], yerr[NVAR];
  double jvs[LU_NZ], rconst[NREACT > 0 ? NREACT : 1], a[NREACT > 0 ? NREACT : 1];
  double b[KPP_NJAC_TMP];
  double k[kMaxStages][NVAR];
  __device__ __forceinline__ Work(double*, long, long) {}
};
#endif

// The environment one cell's rate constants see (the generator's globals).
struct CellEnv {
  double temp, cfactor, sun_fixed;  // sun_fixed < 0: SUN from Update_SUN(TIME)
  double fix[NFIX];
};

__device__ __forceinline__ double cell_sun(const CellEnv& env, double t) {
  return env.sun_fixed >= 0.0 ? env.sun_fixed : kpp_update_sun(t);
}

// Rate constants that stay fixed for the whole integration of a cell: those
// depending only on TEMP/CFACTOR, and the SUN-dependent ones when SUN is
// given per cell.
template <class W>
__device__ __forceinline__ void rates_once(const CellEnv& env, double t, W& w) {
  kpp_rconst_static(w.rconst, t, env.temp, env.cfactor, 0.0, w.y, env.fix);
  if (env.sun_fixed >= 0.0)
    kpp_rconst_sun(w.rconst, t, env.temp, env.cfactor, env.sun_fixed, w.y, env.fix);
}

// Rate constants that change with the time of an evaluation.  The reference
// recomputes all of them at every FunTemplate/JacTemplate call
// (int/rosenbrock.c:1267-1268,1289-1290); recomputing only those whose inputs
// changed gives the same values.
template <class W>
__device__ __forceinline__ bool rates_vary(const CellEnv& env) {
  return KPP_RATES_DYNAMIC > 0 || (KPP_RATES_SUN > 0 && env.sun_fixed < 0.0);
}
template <class W>
__device__ __forceinline__ void rates_at(const CellEnv& env, double t, W& w) {
  if (KPP_RATES_SUN > 0 && env.sun_fixed < 0.0)
    kpp_rconst_sun(w.rconst, t, env.temp, env.cfactor, kpp_update_sun(t), w.y, env.fix);
  if (KPP_RATES_DYNAMIC > 0)
    kpp_rconst_dynamic(w.rconst, t, env.temp, env.cfactor, cell_sun(env, t), w.y, env.fix);
}

// WAXPY (util/blas.c:51-82): y <- y + alpha*x, nothing when alpha == 0.
template <class TX, class TY>
__device__ __forceinline__ void axpy(double alpha, const TX& x, TY& y) {
  if (alpha == 0.0) return;
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) y[i] = y[i] + alpha * x[i];
}

template <class TX, class TY>
__device__ __forceinline__ void copy(const TX& x, TY& y) {
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) y[i] = x[i];
}
