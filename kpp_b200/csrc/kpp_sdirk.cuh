// Batched SDIRK integrator: the reference's C SDIRK (int/sdirk.c, Hairer &
// Wanner's SDIRK4 family: Sdirk2a, 2b, 3a, 4a, 4b) for one cell per thread,
// on the same generated Fun / Jac_SP / LU / solve device code as the
// Rosenbrock kernels.  Included by kpp_rosenbrock.cu in its SDIRK part.
//
// The arithmetic and the control flow are the reference's, operation for
// operation, including the behaviour of its C translation:
//  - controls outside their range print an error in the reference and are
//    then used anyway (SDIRK_ErrorMsg's result is ignored): a negative Hmax,
//    Hmin, Hstart or factor stays 0, a non-positive Newton limit is kept;
//    the tolerance check never stops the run (int/sdirk.c:484-507);
//  - SDIRK_PrepareMatrix gets H, SkipJac and the singularity flag by value:
//    its halving of H on a singular factorisation does not reach the
//    caller, which also never sees the failure (int/sdirk.c:937-989);
//  - a failed Newton iteration shrinks H and then still runs the error
//    estimate and the accept / reject test with the stages computed so far
//    (CycleTloop is reset before it is tested, int/sdirk.c:706-713);
//  - failures (too many steps, step too small) return the caller's Ierr,
//    0, and success returns 1 (int/sdirk.c:599-609, 810-812);
//  - ISTATUS and RSTATUS use the Fortran-style indices 1..8 and 1..3
//    (int/sdirk.c:13-24): here istatus rows 0..7 hold ISTATUS[1..8]
//    (Nfun, Njac, Nstp, Nacc, Nrej, Ndec, Nsol, Nsng) and rstatus rows 0..2
//    hold RSTATUS[1..3] (Texit, Hexit, Hnew), each set at accepted steps.
#pragma once

namespace sdirk {

constexpr int kSmax = 5;

// Method coefficients (int/sdirk.c:994-1312), the published values; only the
// ones the integrator reads.  Theta and Alpha are indexed [j][stage].
struct Method {
  int S;
  double gamma, elo;
  double C[kSmax], D[kSmax], E[kSmax];
  double theta[kSmax][kSmax], alpha[kSmax][kSmax];
};

__constant__ Method c_methods[5] = {
    // Sdirk2a
    {2, 0.2928932188134524755991556378951510, 2.0,
     {0.292893218813452475599155637895151, 1.0},
     {0.0, 1.0},
     {0.4714045207910316829338962414032326, -0.1380711874576983496005629080698993},
     {{0.0, 2.414213562373095048801688724209698}},
     {{0.0, 3.414213562373095048801688724209698}}},
    // Sdirk2b
    {2, 1.707106781186547524400844362104849, 2.0,
     {1.707106781186547524400844362104849, 1.0},
     {0.0, 1.0},
     {-0.4714045207910316829338962414032326, 0.8047378541243650162672295747365659},
     {{0.0, -0.414213562373095048801688724209698}},
     {{0.0, 0.5857864376269049511983112757903019}}},
    // Sdirk3a
    {3, 0.2113248654051871177454256097490213, 2.0,
     {0.2113248654051871177454256097490213, 0.4226497308103742354908512194980427, 1.0},
     {0.0, 0.0, 1.0},
     {0.9106836025229590978424821138352906, -1.244016935856292431175815447168624,
      0.3333333333333333333333333333333333},
     {{0.0, 1.0, -1.732050807568877293527446341505872},
      {0.0, 0.0, 2.732050807568877293527446341505872}},
     {{0.0, 2.0, -12.92820323027550917410978536602349},
      {0.0, 0.0, 8.83012701892219323381861585376468}}},
    // Sdirk4a
    {5, 0.2666666666666666666666666666666667, 4.0,
     {0.2666666666666666666666666666666667, 0.7666666666666666666666666666666667,
      0.5666666666666666666666666666666667, 0.3661315380631796996374935266701191, 1.0},
     {0.0, 0.0, 0.0, 0.0, 1.0},
     {-0.6804000050475287124787034884002302, 1.558961944525217193393931795738823,
      -13.55893003128907927748632408763868, 15.48522576958521253098585004571302, 1.0},
     {{0.0, 1.875000000000000000000000000000000, 1.708847304091539528432732316227462,
       0.2680325578937783958847157206823118, 0.9096171815241460655379433581446771},
      {0.0, 0.0, -0.2030773231622746185852981969486824, -0.1828840955527181631794050728644549,
       -3.108254967778352416114774430509465},
      {0.0, 0.0, 0.0, 0.2968246986151577397160821594427966, 12.33727431701306195581826123274001},
      {0.0, 0.0, 0.0, 0.0, -11.24557012450885560524143016037523}},
     {{0.0, 2.875000000000000000000000000000000, 0.8500000000000000000000000000000000,
       0.7352046091658870564637910527807370, -16.10898993405067684831655675112808},
      {0.0, 0.0, 0.4434782608695652173913043478260870, -0.9525565003057343527941920657462074e-01,
       6.559571569643355712998131800797873},
      {0.0, 0.0, 0.0, 0.4290111305453813852259481840631738, -15.90772144271326504260996815012482},
      {0.0, 0.0, 0.0, 0.0, 25.34908987169226073668861694892683}}},
    // Sdirk4b
    {5, 0.25, 4.0,
     {0.25, 0.75, 0.55, 0.5, 1.0},
     {0.0, 0.0, 0.0, 0.0, 1.0},
     {0.5750, 0.2125, -4.6875, 4.2500, 0.1500},
     {{0.0, 2.0, 1.680000000000000000000000000000000, 1.308823529411764705882352941176471,
       -3.083333333333333333333333333333333},
      {0.0, 0.0, -0.1600000000000000000000000000000000, -0.1838235294117647058823529411764706,
       -4.291666666666666666666666666666667},
      {0.0, 0.0, 0.0, 0.1102941176470588235294117647058824, 34.37500000000000000000000000000000},
      {0.0, 0.0, 0.0, 0.0, -28.3333333333333333333333333333}},
     {{0.0, 3.0, 0.8800000000000000000000000000000000, 0.1666666666666666666666666666666667,
       -6.0},
      {0.0, 0.0, 0.4400000000000000000000000000000000, -0.8333333333333333333333333333333333e-01,
       9.0},
      {0.0, 0.0, 0.0, 0.9469696969696969696969696969696970, -56.81818181818181818181818181818182},
      {0.0, 0.0, 0.0, 0.0, 54.0}}},
};

// ICNTRL[2] -> method: 1 Sdirk2a, 2 Sdirk2b, 3 Sdirk3a, 4 Sdirk4a, 5 Sdirk4b,
// anything else Sdirk2a (int/sdirk.c:296-318).
__device__ __forceinline__ int method_index(int icntrl2) {
  return (icntrl2 >= 2 && icntrl2 <= 5) ? icntrl2 - 1 : 0;
}

// Per-cell work arrays: Z[S], G, TMP, RHS, SCAL, the Jacobian FJAC (kept
// between steps for SkipJac) and the factorised E, rate constants and the
// Fun / Jac_SP temporaries.
constexpr long kPerSlot = kSdirkPerSlot;
static_assert(kSdirkStages == kSmax, "stage count of the work layout");

#if defined(KPP_SCRATCH)
struct Work {
  Strided y, g, tmp, rhs, scal, fjac, e, rconst, a, b;
  Strided z[kSmax];
  __device__ __forceinline__ Work(double* base, long slot) {
    double* block = base + (slot / kLanes) * kPerSlot * kLanes + (slot % kLanes);
    long off = 0;
    auto take = [&](long n) {
      Strided v{block + off * kLanes};
      off += n;
      return v;
    };
    y = take(NVAR); g = take(NVAR); tmp = take(NVAR); rhs = take(NVAR); scal = take(NVAR);
    fjac = take(LU_NZ); e = take(LU_NZ); rconst = take(NREACT); a = take(NREACT);
    b = take(KPP_NJAC_TMP);
    for (int s = 0; s < kSmax; s++) z[s] = take(NVAR);
  }
};
#else
struct Work {
  double y[NVAR], g[NVAR], tmp[NVAR], rhs[NVAR], scal[NVAR];
  double fjac[LU_NZ], e[LU_NZ], rconst[NREACT > 0 ? NREACT : 1], a[NREACT > 0 ? NREACT : 1];
  double b[KPP_NJAC_TMP];
  double z[kSmax][NVAR];
  __device__ __forceinline__ Work(double*, long) {}
};
#endif

// SIGN(x, y) of int/sdirk.c:5: ((x*y) >= 0 ? x : -x)
__device__ __forceinline__ double sd_sign(double x, double y) { return (x * y >= 0) ? x : -x; }

// WSCAL (util/blas.c:86-): x <- alpha x, nothing for alpha == 1, zeros for 0.
template <class T>
__device__ __forceinline__ void wscal(double alpha, T& x) {
  if (alpha == 1.0) return;
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) x[i] = (alpha == 0.0) ? 0.0 : alpha * x[i];
}

// SDIRK_ErrorScale (int/sdirk.c:815-834)
template <class W>
__device__ __forceinline__ void error_scale(W& w, const double* atol, const double* rtol,
                                            bool scalar_tol) {
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) {
    const double a = scalar_tol ? atol[0] : atol[i], r = scalar_tol ? rtol[0] : rtol[i];
    w.scal[i] = 1.0 / (a + r * ros_abs(w.y[i]));
  }
}

// SDIRK_ErrorNorm (int/sdirk.c:837-851): sqrt(mean((y scal)^2)), at least
// 1e-10; pow(x, 2) and pow(x, 0.5) of the reference are the correctly
// rounded square and square root.
template <class TY, class TS>
__device__ __forceinline__ double error_norm(const TY& y, const TS& scal) {
  double err = 0.0;
#pragma unroll 4
  for (int i = 0; i < NVAR; i++) {
    const double v = y[i] * scal[i];
    err = err + v * v;
  }
  const double r = sqrt(err / (double)NVAR);
  return r >= 1.0e-10 ? r : 1.0e-10;
}

// SDIRK_Solve (int/sdirk.c:992-1012): rhs <- (1/(H gamma)) rhs, then the LU
// solve with E.
template <class W>
__device__ __forceinline__ void solve(double h, double gamma, W& w, int which, Stats& st) {
  const double hgi = 1.0 / (h * gamma);
  if (which == 0) {
    wscal(hgi, w.rhs);
    kpp_solve(w.e, w.rhs);
  } else {
    wscal(hgi, w.tmp);
    kpp_solve(w.e, w.tmp);
  }
  st.nsol++;
}

// SDIRK_PrepareMatrix (int/sdirk.c:937-989) with its arguments by value.
template <class W>
__device__ __forceinline__ void prepare_matrix(const CellEnv& env, double h, double t,
                                               double gamma, bool skip_jac, W& w, Stats& st) {
  int consecutive = 0;
  int ising = 1;
  while (ising != 0) {
    const double hgi = 1.0 / (h * gamma);
    if (!skip_jac) {
      // JAC_CHEM(T, Y, FJAC) (int/sdirk.c:1329-1360)
      if (rates_vary<W>(env)) rates_at(env, t, w);
      kpp_jac_sp<false>(w.y, env.fix, w.rconst, w.fjac, w.b);
      st.njac++;
    }
#pragma unroll 4
    for (int i = 0; i < LU_NZ; i++) w.e[i] = -w.fjac[i];
    kpp_add_diagonal(w.e, hgi);
    ising = kpp_decomp(w.e, w.tmp);  // tmp is free here: the work row
    st.ndec++;
    if (ising != 0) {
      st.nsng++;
      consecutive++;
      if (consecutive >= 6) return;
      h = 0.5 * h;
      skip_jac = true;
    }
  }
}

// SDIRK_Integrator (int/sdirk.c:513-812).  Returns 1 or 0 (see above).
template <class W>
__device__ int integrate(const CellEnv& env, W& w, const Method& m, double tinit, double tfinal,
                         double hstart, double hmin, double hmax, const double* atol,
                         const double* rtol, bool scalar_tol, int max_no_steps,
                         bool start_newton, double newton_tol, double theta_min, double facsafe,
                         double facmin, double facmax, double facrej, double qmin, double qmax,
                         int newton_maxit, double rst[3], Stats& st) {
  const double roundoff = kRoundoff;
  double t = tinit;
  const double tdir = sd_sign(1.0, tfinal - tinit);
  double h = ros_max(ros_abs(hmin), ros_abs(hstart));
  if (ros_abs(h) <= 10.0 * roundoff) h = 1.0e-06;
  h = ros_min(ros_abs(h), hmax);
  h = sd_sign(h, tdir);
  bool skip_lu = false, skip_jac = false, reject = false, first_step = true;
  double theta = 0.0, newton_increment_old = 0.0;
  const int S = m.S;
  // The stage vectors start at zero.  After a Newton failure the reference
  // still runs the error estimate of the step (CycleTloop is reset before
  // it is tested, int/sdirk.c:700-713), which reads Z of the stages the step
  // did not reach: the previous step's values or, in the first step, a local
  // array of SDIRK_Integrator (:516) not yet written; zero here, as a fresh
  // stack frame holds.
  for (int s = 0; s < kSmax; s++) {
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.z[s][i] = 0.0;
  }
  rates_once(env, t, w);
  error_scale(w, atol, rtol, scalar_tol);

  while ((tfinal - t) * tdir - roundoff > 0.0) {
    if (!skip_lu) prepare_matrix(env, h, t, m.gamma, skip_jac, w, st);
    if (st.nstp > max_no_steps) return 0;
    if ((t + 0.1 * h == t) || (ros_abs(h) <= roundoff)) return 0;

    for (int istage = 0; istage < S; istage++) {
#pragma unroll 4
      for (int i = 0; i < NVAR; i++) {
        w.z[istage][i] = 0.0;
        w.g[i] = 0.0;
      }
      for (int j = 0; j < istage; j++) {
        axpy(m.theta[j][istage], w.z[j], w.g);
        if (start_newton) axpy(m.alpha[j][istage], w.z[j], w.z[istage]);
      }
      bool newton_done = false;
      double fac = 0.5;
      double newton_rate = 0.0;
      for (int it = 0; it < newton_maxit; it++) {
#pragma unroll 4
        for (int i = 0; i < NVAR; i++) w.tmp[i] = w.y[i] + w.z[istage][i];
        // FUN_CHEM(T + C H, TMP, RHS) (int/sdirk.c:1314-1327)
        if (rates_vary<W>(env)) rates_at(env, t + m.C[istage] * h, w);
        kpp_fun(w.tmp, env.fix, w.rconst, w.rhs, w.a);
        st.nfun++;
        wscal(h * m.gamma, w.rhs);
        axpy(-1.0, w.z[istage], w.rhs);
        axpy(1.0, w.g, w.rhs);
        solve(h, m.gamma, w, 0, st);
        const double newton_increment = error_norm(w.rhs, w.scal);
        if (it == 0) {
          theta = ros_abs(theta_min);
          newton_rate = 2.0;
        } else {
          theta = newton_increment / newton_increment_old;
          if (theta < 0.99) {
            newton_rate = theta / (1.0 - theta);
            const double predicted =
                newton_increment * KPP_POW(theta, (newton_maxit - (it + 1)) / (1.0 - theta));
            if (predicted >= newton_tol) {
              const double qn = ros_min(10.0, predicted / newton_tol);
              fac = 0.8 * KPP_POW(qn, (-1.0 / (1 + newton_maxit - it + 1)));
              break;
            }
          } else {
            break;
          }
        }
        newton_increment_old = newton_increment;
        axpy(1.0, w.rhs, w.z[istage]);
        newton_done = (newton_rate * newton_increment <= newton_tol);
        if (newton_done) break;
      }
      if (!newton_done) {
        h = fac * h;
        reject = true;
        skip_jac = true;
        skip_lu = false;
        break;  // CycleTloop, reset before its test: the step goes on below
      }
    }

    // error estimation (int/sdirk.c:716-733)
    st.nstp++;
#pragma unroll 4
    for (int i = 0; i < NVAR; i++) w.tmp[i] = 0.0;
    for (int i = 0; i < S; i++)
      if (m.E[i] != 0.0) axpy(m.E[i], w.z[i], w.tmp);
    solve(h, m.gamma, w, 1, st);
    const double err = error_norm(w.tmp, w.scal);
    double fac = facsafe * KPP_POW(err, (-1.0 / m.elo));
    fac = ros_max(facmin, ros_min(facmax, fac));
    double hnew = h * fac;

    if (err < 1.0) {  // accept
      first_step = false;
      st.nacc++;
      t = t + h;
      for (int i = 0; i < S; i++)
        if (m.D[i] != 0.0) axpy(m.D[i], w.z[i], w.y);
      error_scale(w, atol, rtol, scalar_tol);
      hnew = tdir * ros_min(ros_abs(hnew), hmax);
      rst[0] = t;
      rst[1] = h;
      rst[2] = hnew;
      if (reject) hnew = tdir * ros_min(ros_abs(hnew), ros_abs(h));
      reject = false;
      if ((t + hnew / qmin - tfinal) * tdir > 0.0) {
        h = tfinal - t;
      } else {
        const double hratio = hnew / h;
        skip_lu = (theta <= theta_min) && (hratio >= qmin) && (hratio <= qmax);
        if (!skip_lu) h = hnew;
      }
      skip_jac = false;
    } else {  // reject
      if (first_step || reject) h = facrej * h;
      else h = hnew;
      reject = true;
      skip_jac = true;
      skip_lu = false;
      if (st.nacc >= 1) st.nrej++;
    }
  }
  return 1;
}

// SDIRK (int/sdirk.c:170-511): controls as the reference reads them, then
// the integrator.
template <class W>
__device__ int sdirk_cell(const CellEnv& env, W& w, double tinit, double tfinal,
                          const double* atol, const double* rtol, const int* icntrl,
                          const double* rcntrl, double rst[3], Stats& st) {
  const Method& m = c_methods[method_index(icntrl[2])];
  const bool scalar_tol = icntrl[1] != 0;  // ITOL = 0
  const int max_no_steps = icntrl[3] == 0 ? 200000 : (icntrl[3] > 0 ? icntrl[3] : 0);
  const int newton_maxit = icntrl[4] == 0 ? 8 : icntrl[4];
  const bool start_newton = icntrl[5] == 0;
  const double span = ros_abs_diff(tfinal, tinit);
  const double hmin = rcntrl[0] > 0.0 ? rcntrl[0] : 0.0;
  const double hmax = rcntrl[1] == 0.0 ? span : (rcntrl[1] > 0.0 ? ros_min(ros_abs(rcntrl[1]), span)
                                                                  : 0.0);
  const double hstart = rcntrl[2] == 0.0 ? ros_max(hmin, kRoundoff)
                                         : (rcntrl[2] > 0.0 ? ros_min(ros_abs(rcntrl[2]), span)
                                                            : 0.0);
  const double facmin = rcntrl[3] == 0.0 ? 0.2 : (rcntrl[3] > 0.0 ? rcntrl[3] : 0.0);
  const double facmax = rcntrl[4] == 0.0 ? 10.0 : (rcntrl[4] > 0.0 ? rcntrl[4] : 0.0);
  const double facrej = rcntrl[5] == 0.0 ? 0.1 : (rcntrl[5] > 0.0 ? rcntrl[5] : 0.0);
  const double facsafe = rcntrl[6] == 0.0 ? 0.9 : (rcntrl[6] > 0.0 ? rcntrl[6] : 0.0);
  const double theta_min = rcntrl[7] == 0.0 ? 1.0e-03 : rcntrl[7];
  const double newton_tol = rcntrl[8] == 0.0 ? 3.0e-02 : rcntrl[8];
  const double qmin = rcntrl[9] == 0.0 ? 1.0 : rcntrl[9];
  const double qmax = rcntrl[10] == 0.0 ? 1.2 : rcntrl[10];
  return integrate(env, w, m, tinit, tfinal, hstart, hmin, hmax, atol, rtol, scalar_tol,
                   max_no_steps, start_newton, newton_tol, theta_min, facsafe, facmin, facmax,
                   facrej, qmin, qmax, newton_maxit, rst, st);
}

}  // namespace sdirk
