// The Rosenbrock discrete adjoint of int/rosenbrock_adj.c (RosenbrockADJ,
// :191-597), one cell per thread: the forward integration with its
// trajectory kept per cell (ros_FwdInt and ros_DPush, :949-1173, :779-815),
// then the backward pass over it (ros_DadjInt and ros_DPop, :1177-1318,
// :817-855), for NADJ adjoint vectors Lambda of every cell.
//
// The mechanism functions are the ones KPP's own generator writes with
// #LANGUAGE CUDA and #HESSIAN ON (kpp_b200/kppgen): Update_RCONST, Fun,
// Jac_SP, Hessian, HessTR_Vec, JacTR_SP_Vec, KppDecomp, KppSolve and
// KppSolveTR, called on strided views of the cell's arrays.  Compiled for
// the host by tests/host_adj.cpp, the same code is compared bit for bit with
// the reference's RosenbrockADJ; on the device it runs in the
// generator-route library (kpp_rosenbrock.cu, KPP_PART 8).
//
// The reference's semantics kept, including the ones that differ from
// int/rosenbrock.c: DeltaMin = 1e-5; the tableaux of rosenbrock_adj.c (Ros2
// with g = 1 + 1/SQRT(2) computed, Rodas3's C(4,3) = -(8/3), Rodas3_1
// selectable as method 7); Hstart = MIN(MAX(|Hmin|, |Hstart|), |Hmax|) and a
// signed H; ros_PrepareMatrix halving only its own copy of H; the error norm
// as SQRT of the mean of pow(Yerr/Scale, 2), at least 1e-10; any nonzero
// ICNTRL[3] rejected (-1: the reference compares its still-zero local
// Max_no_steps), the step limit being bufsize - 1; the backward loop
// `while (stack_ptr > 0)`, which leaves the first accepted step out of the
// adjoint.  SQRT and pow are KPP_POW (correctly rounded on the device; the
// C library's in the host build).
#pragma once

namespace kpp_adj {

constexpr double kAdjDeltaMin = 1.0e-5;  // rosenbrock_adj.c: DeltaMin

// One cell's column of a structure-of-arrays buffer: element i at p[i*ld].
struct Col {
  double* p;
  long ld;
  __host__ __device__ __forceinline__ double& operator[](long i) const { return p[i * ld]; }
  __host__ __device__ __forceinline__ Col at(long off) const { return Col{p + off * ld, ld}; }
};

// Tableaux of rosenbrock_adj.c (:2054-2470): ros_S, A, C, M, E, Alpha,
// Gamma, ELO and NewF; A and C strictly lower triangular, row-wise.
struct AdjTableau {
  int S;
  double A[15], C[15], M[6], E[6], Alpha[6], Gamma[6], ELO;
  bool NewF[6];
};

// method: 1 Ros2, 2 Ros3, 3 Ros4, 4 Rodas3, 5 Rodas4, 7 Rodas3_1.
__host__ __device__ inline AdjTableau adj_tableau(int method) {
  AdjTableau t{};
  if (method == 2 || method == 3 || method == 5) {
    // the coefficients of int/rosenbrock.c, the same numbers here
    const Tableau r = make_tableau(method);
    t.S = r.S;
    for (int i = 0; i < 15; i++) {
      t.A[i] = r.A[i];
      t.C[i] = r.C[i];
    }
    for (int i = 0; i < 6; i++) {
      t.M[i] = r.M[i];
      t.E[i] = r.E[i];
      t.Alpha[i] = r.Alpha[i];
      t.Gamma[i] = r.Gamma[i];
      t.NewF[i] = r.NewF[i];
    }
    t.ELO = r.ELO;
  } else if (method == 1) {  // Ros2, g = 1 + 1/sqrt(2) evaluated
    const double g = 1.0 + 1.0 / 1.4142135623730951;
    t.S = 2;
    t.A[0] = 1.0 / g;
    t.C[0] = (-2.0) / g;
    t.NewF[0] = true;
    t.NewF[1] = true;
    t.M[0] = 3.0 / (2.0 * g);
    t.M[1] = 1.0 / (2.0 * g);
    t.E[0] = 1.0 / (2.0 * g);
    t.E[1] = 1.0 / (2.0 * g);
    t.ELO = 2.0;
    t.Alpha[0] = 0.0;
    t.Alpha[1] = 1.0;
    t.Gamma[0] = g;
    t.Gamma[1] = -g;
  } else if (method == 4) {  // Rodas3
    t.S = 4;
    t.A[0] = 0.0; t.A[1] = 2.0; t.A[2] = 0.0; t.A[3] = 2.0; t.A[4] = 0.0; t.A[5] = 1.0;
    t.C[0] = 4.0; t.C[1] = 1.0; t.C[2] = -1.0; t.C[3] = 1.0; t.C[4] = -1.0;
    t.C[5] = -(8.0 / 3.0);
    t.NewF[0] = true; t.NewF[1] = false; t.NewF[2] = true; t.NewF[3] = true;
    t.M[0] = 2.0; t.M[1] = 0.0; t.M[2] = 1.0; t.M[3] = 1.0;
    t.E[0] = 0.0; t.E[1] = 0.0; t.E[2] = 0.0; t.E[3] = 1.0;
    t.ELO = 3.0;
    t.Alpha[0] = 0.0; t.Alpha[1] = 0.0; t.Alpha[2] = 1.0; t.Alpha[3] = 1.0;
    t.Gamma[0] = 0.5; t.Gamma[1] = 1.5; t.Gamma[2] = 0.0; t.Gamma[3] = 0.0;
  } else if (method == 7) {  // Rodas3_1
    t.S = 4;
    t.A[0] = 0.0; t.A[1] = 1.5382237953138116; t.A[2] = -0.36440683885434433;
    t.A[3] = 1.538223795313811; t.A[4] = -0.36440683885434433; t.A[5] = 1.0;
    t.C[0] = -4.0919303685081028; t.C[1] = -3.0551174378039538e-002;
    t.C[2] = 1.7259281281917580; t.C[3] = 0.19561160936073679;
    t.C[4] = 1.9301670595355112; t.C[5] = -2.6267006001193960;
    t.NewF[0] = true; t.NewF[1] = false; t.NewF[2] = true; t.NewF[3] = true;
    t.M[0] = 1.5382237953138116; t.M[1] = -0.36440683885434444;
    t.M[2] = 1.0000000000000002; t.M[3] = 1.0;
    t.E[0] = 0.0; t.E[1] = 0.0; t.E[2] = 0.0; t.E[3] = 1.0;
    t.ELO = 3.0;
    t.Alpha[0] = 0.0; t.Alpha[1] = 0.0; t.Alpha[2] = 1.0; t.Alpha[3] = 1.0;
    t.Gamma[0] = 0.5150000000000000; t.Gamma[1] = -0.57028223198756145;
    t.Gamma[2] = 0.0; t.Gamma[3] = 0.0;
  }
  return t;
}

// util/blas.c's WAXPY and WSCAL over n elements, with their special cases
// (alpha 0: no-op / zero fill; alpha 1: no-op; alpha -1: negation).
template <class TX, class TY>
__host__ __device__ __forceinline__ void waxpy(int n, double alpha, const TX& x, TY& y) {
  if (alpha == 0.0) return;
  for (int i = 0; i < n; i++) y[i] = y[i] + alpha * x[i];
}
template <class TX>
__host__ __device__ __forceinline__ void wscal(int n, double alpha, TX& x) {
  if (alpha == 1.0) return;
  for (int i = 0; i < n; i++) x[i] = (alpha == -1.0) ? -x[i] : (alpha == 0.0 ? 0.0 : alpha * x[i]);
}
template <class TX, class TY>
__host__ __device__ __forceinline__ void wcopy(int n, const TX& x, TY& y) {
  for (int i = 0; i < n; i++) y[i] = x[i];
}

// Offsets (in elements of a cell's column) of the work arrays and the
// trajectory of one cell; the stage arrays are sized for 6 stages.
struct AdjLayout {
  long rconst, ynew, fcn0, fcn, dfdt, yerr, tmp, tmp2, k, ystage, jac0, ghimj, jac, djdt, hes,
      u, v, traj, entry, total;
};

__host__ __device__ inline AdjLayout adj_layout(int nadj, int bufsize, bool save_lu) {
  AdjLayout L{};
  long o = 0;
  L.rconst = o; o += KPP_NREACT;
  L.ynew = o; o += NVAR;
  L.fcn0 = o; o += NVAR;
  L.fcn = o; o += NVAR;
  L.dfdt = o; o += NVAR;
  L.yerr = o; o += NVAR;
  L.tmp = o; o += NVAR;
  L.tmp2 = o; o += NVAR;
  L.k = o; o += 6L * NVAR;
  L.ystage = o; o += 6L * NVAR;
  L.jac0 = o; o += LU_NZ;
  L.ghimj = o; o += LU_NZ;
  L.jac = o; o += LU_NZ;
  L.djdt = o; o += LU_NZ;
  L.hes = o; o += KPP_NHESS;
  L.u = o; o += (long)nadj * 6 * NVAR;
  L.v = o; o += (long)nadj * 6 * NVAR;
  // one trajectory entry: T, H, the stage states, the stage vectors and,
  // with SaveLU, the factorised matrix (ros_DPush, :779-815)
  L.entry = 2 + 12L * NVAR + (save_lu ? (long)LU_NZ : 0L);
  L.traj = o; o += (long)bufsize * L.entry;
  L.total = o;
  return L;
}

// The controls of RosenbrockADJ (:191-520) for a call over [tstart, tend].
struct AdjControls {
  bool autonomous, vectortol, save_lu, discrete;
  int method, max_no_steps;
  double hmin, hmax, hstart, facmin, facmax, facrej, facsafe;
};

// Validation and defaults in the reference's order; 0, or its IERR.
// adjoint_type: ICNTRL[6] as given (0 = discrete).
__device__ inline int adj_controls(const int* icntrl, const double* rcntrl, const double* atol,
                                   const double* rtol, int bufsize, double tstart, double tend,
                                   AdjControls& c) {
  c.autonomous = !(icntrl[0] == 0);
  c.vectortol = (icntrl[1] == 0);
  const int uplimtol = c.vectortol ? NVAR : 1;
  switch (icntrl[2]) {
    case 0:
    case 4: c.method = 4; break;
    case 1: c.method = 1; break;
    case 2: c.method = 2; break;
    case 3: c.method = 3; break;
    case 5: c.method = 5; break;
    case 7: c.method = 7; break;
    default: return -2;
  }
  // ICNTRL[3] != 0 is rejected: the reference tests its local Max_no_steps,
  // still 0, instead of ICNTRL[3] (:410-416)
  if (icntrl[3] == 0) c.max_no_steps = bufsize - 1;
  else return -1;
  if (!(icntrl[5] == 0 || (icntrl[5] >= 1 && icntrl[5] <= 5))) return -2;
  if (!(icntrl[6] == 0 || (icntrl[6] >= 1 && icntrl[6] <= 4))) return -9;
  c.discrete = (icntrl[6] == 0 || icntrl[6] == 2);
  c.save_lu = (icntrl[7] != 0);
  if (rcntrl[0] == 0.0) c.hmin = 0.0;
  else if (rcntrl[0] > 0.0) c.hmin = rcntrl[0];
  else return -3;
  if (rcntrl[1] == 0.0) c.hmax = ros_abs_diff(tend, tstart);
  else if (rcntrl[1] > 0.0) c.hmax = ros_min(ros_abs(rcntrl[1]), ros_abs_diff(tend, tstart));
  else return -3;
  if (rcntrl[2] == 0.0) c.hstart = ros_max(c.hmin, kAdjDeltaMin);
  else if (rcntrl[2] > 0.0) c.hstart = ros_min(ros_abs(rcntrl[2]), ros_abs_diff(tend, tstart));
  else return -3;
  if (rcntrl[3] == 0.0) c.facmin = 0.2;
  else if (rcntrl[3] > 0.0) c.facmin = rcntrl[3];
  else return -4;
  if (rcntrl[4] == 0.0) c.facmax = 6.0;
  else if (rcntrl[4] > 0.0) c.facmax = rcntrl[4];
  else return -4;
  if (rcntrl[5] == 0.0) c.facrej = 0.1;
  else if (rcntrl[5] > 0.0) c.facrej = rcntrl[5];
  else return -4;
  if (rcntrl[6] == 0.0) c.facsafe = 0.9;
  else if (rcntrl[6] > 0.0) c.facsafe = rcntrl[6];
  else return -4;
  for (int i = 0; i < uplimtol; i++)
    if ((atol[i] <= 0.0) || (rtol[i] <= 10.0 * kRoundoff) || (rtol[i] >= 1.0)) return -5;
  return 0;
}

// Statistics and exit values of one cell: ISTATUS[1..8] and RSTATUS[1..3]
// (Texit, Hexit, Hnew) of the reference.
struct AdjStatus {
  int nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng;
  double texit, hexit, hnew;
};

// FunTemplate / JacTemplate / HessTemplate (:2474-2544): Update_SUN and
// Update_RCONST at time t (their species are the generator's global C, the
// cell's VAR, which the forward pass integrates in place), then the function.
__device__ __forceinline__ void adj_rates(const CellEnv& env, double t, const Col& var,
                                          Col rconst) {
  kpp_update_rconst(rconst, t, env.temp, env.cfactor, cell_sun(env, t), var, env.fix);
}

// ros_ErrorNorm (:1747-1771)
__device__ __forceinline__ double adj_error_norm(const Col& y, const Col& ynew, const Col& yerr,
                                                 const double* atol, const double* rtol,
                                                 bool vectortol) {
  double err = 0.0;
  for (int i = 0; i < NVAR; i++) {
    const double ymax = ros_max(ros_abs(y[i]), ros_abs(ynew[i]));
    const double scale = vectortol ? (atol[i] + rtol[i] * ymax) : (atol[0] + rtol[0] * ymax);
    const double q = yerr[i] / scale;
    err = err + q * q;  // pow(q, 2): the C compiler folds it into q*q
  }
  err = KPP_POW(err / NVAR, 0.5);  // SQRT(x) is pow(x, 0.5) (:4)
  return ros_max(err, 1.0e-10);
}

// ros_PrepareMatrix (:1813-1873): Ghimj = -Jac0 + 1/(Direction H gam) I,
// factorised; H is the function's own copy (halved on a singular matrix,
// at most 5 times).  Returns true when the matrix stays singular.
__device__ __forceinline__ bool adj_prepare_matrix(double h, int direction, double gam,
                                                   const Col& jac0, Col& ghimj, AdjStatus& st) {
  int nconsecutive = 0;
  for (;;) {
    wcopy(LU_NZ, jac0, ghimj);
    wscal(LU_NZ, -1.0, ghimj);
    const double ghinv = 1.0 / (direction * h * gam);
    for (int i = 0; i < NVAR; i++) ghimj[LU_DIAG[i]] = ghimj[LU_DIAG[i]] + ghinv;
    const int ising = KppDecomp(ghimj);
    st.ndec++;
    if (ising == 0) return false;
    st.nsng++;
    nconsecutive++;
    if (nconsecutive <= 5) h = h * 0.5;
    else return true;
  }
}

// ros_FwdInt (:949-1173) with the discrete adjoint's checkpoints: each
// accepted step pushes T, H, the stage states, the stage vectors and (SaveLU)
// the factorised matrix into the cell's trajectory.  Returns IERR; *npush =
// the entries pushed.
__device__ inline int adj_forward(const CellEnv& env, const AdjControls& c, const AdjTableau& tab,
                                  const double* atol, const double* rtol, double tstart,
                                  double tend, Col y, Col w, const AdjLayout& L, int& npush,
                                  AdjStatus& st) {
  Col rconst = w.at(L.rconst), ynew = w.at(L.ynew), fcn0 = w.at(L.fcn0), fcn = w.at(L.fcn),
      dfdt = w.at(L.dfdt), yerr = w.at(L.yerr), k = w.at(L.k), ystage = w.at(L.ystage),
      jac0 = w.at(L.jac0), ghimj = w.at(L.ghimj);
  const int S = tab.S;
  double t = tstart;
  st.hexit = 0.0;
  double h = ros_min(ros_max(ros_abs(c.hmin), ros_abs(c.hstart)), ros_abs(c.hmax));
  if (ros_abs(h) <= 10.0 * kRoundoff) h = kAdjDeltaMin;
  const int direction = (tend >= tstart) ? 1 : -1;
  h = direction * h;
  bool reject_last = false, reject_more = false;
  npush = 0;
  while (((direction > 0) && ((t - tend) + kRoundoff <= 0.0)) ||
         ((direction < 0) && ((tend - t) + kRoundoff <= 0.0))) {
    if (st.nstp > c.max_no_steps) return -6;
    if (((t + 0.1 * h) == t) || (h <= kRoundoff)) return -7;
    st.hexit = h;
    h = ros_min(h, ros_abs_diff(tend, t));
    adj_rates(env, t, y, rconst);
    Fun(y, env.fix, rconst, fcn0);
    st.nfun++;
    if (!c.autonomous) {
      // ros_FunTimeDerivative (:1773-1789)
      const double delta = KPP_POW(kRoundoff, 0.5) * ros_max(kAdjDeltaMin, ros_abs(t));
      adj_rates(env, t + delta, y, rconst);
      Fun(y, env.fix, rconst, dfdt);
      st.nfun++;
      waxpy(NVAR, -1.0, fcn0, dfdt);
      wscal(NVAR, 1.0 / delta, dfdt);
    }
    adj_rates(env, t, y, rconst);
    Jac_SP(y, env.fix, rconst, jac0);
    st.njac++;
    for (;;) {  // UntilAccepted
      if (adj_prepare_matrix(h, direction, tab.Gamma[0], jac0, ghimj, st)) return -8;
      for (int is = 0; is < S; is++) {
        Col ks = k.at((long)NVAR * is);
        if (is == 0) {
          wcopy(NVAR, fcn0, fcn);
          if (c.discrete) {
            wcopy(NVAR, y, ystage);
            wcopy(NVAR, y, ynew);
          }
        } else if (tab.NewF[is]) {
          wcopy(NVAR, y, ynew);
          for (int j = 0; j < is; j++)
            waxpy(NVAR, tab.A[is * (is - 1) / 2 + j], k.at((long)NVAR * j), ynew);
          const double tau = t + tab.Alpha[is] * direction * h;
          adj_rates(env, tau, y, rconst);
          Fun(ynew, env.fix, rconst, fcn);
          st.nfun++;
        }
        if (is > 0 && c.discrete) {
          Col yst = ystage.at((long)NVAR * is);
          wcopy(NVAR, ynew, yst);
        }
        wcopy(NVAR, fcn, ks);
        for (int j = 0; j < is; j++) {
          const double hc = tab.C[is * (is - 1) / 2 + j] / (direction * h);
          waxpy(NVAR, hc, k.at((long)NVAR * j), ks);
        }
        if ((!c.autonomous) && (tab.Gamma[is] != 0.0)) {
          const double hg = direction * h * tab.Gamma[is];
          waxpy(NVAR, hg, dfdt, ks);
        }
        KppSolve(ghimj, ks);
        st.nsol++;
      }
      wcopy(NVAR, y, ynew);
      for (int j = 0; j < S; j++) waxpy(NVAR, tab.M[j], k.at((long)NVAR * j), ynew);
      wscal(NVAR, 0.0, yerr);
      for (int j = 0; j < S; j++) waxpy(NVAR, tab.E[j], k.at((long)NVAR * j), yerr);
      const double err = adj_error_norm(y, ynew, yerr, atol, rtol, c.vectortol);
      const double fac =
          ros_min(c.facmax, ros_max(c.facmin, c.facsafe / KPP_POW(err, 1.0 / tab.ELO)));
      double hnew = h * fac;
      st.nstp++;
      if ((err <= 1.0) || (h <= c.hmin)) {
        st.nacc++;
        if (c.discrete) {  // ros_DPush
          Col e = w.at(L.traj + (long)npush * L.entry);
          e[0] = h;
          e[1] = t;
          for (int i = 0; i < NVAR * S; i++) {
            e[2 + i] = ystage[i];
            e[2 + 6L * NVAR + i] = k[i];
          }
          if (c.save_lu)
            for (int i = 0; i < LU_NZ; i++) e[2 + 12L * NVAR + i] = ghimj[i];
          npush++;
        }
        wcopy(NVAR, ynew, y);
        t = t + direction * h;
        hnew = ros_max(c.hmin, ros_min(hnew, c.hmax));
        if (reject_last) hnew = ros_min(hnew, h);
        st.hexit = h;
        st.hnew = hnew;
        st.texit = t;
        reject_last = false;
        reject_more = false;
        h = hnew;
        break;
      }
      if (reject_more) hnew = h * c.facrej;
      reject_more = reject_last;
      reject_last = true;
      h = hnew;
      if (st.nacc >= 1) st.nrej++;
    }
  }
  return 1;
}

// ros_DadjInt (:1177-1318): the pushed steps, last first, down to the
// second (`while (stack_ptr > 0)`): per step the LU of Ghimj (saved, or
// recomputed from the Jacobian at the step's start), the Hessian there, the
// stage adjoints U (transposed solves) and V = Jac(T_i, Y_i)^T U, and Lambda
// += sum V_i + (H0 x K_i)^T U_i (+ H dJ/dT^T sum gamma_i U_i when the
// system depends on time).  lambda holds NADJ vectors of NVAR, in place.
__device__ inline int adj_backward(const CellEnv& env, const AdjControls& c,
                                   const AdjTableau& tab, double tstart, double tend, Col y,
                                   Col lambda, int nadj, Col w, const AdjLayout& L, int npush,
                                   AdjStatus& st) {
  Col rconst = w.at(L.rconst), tmp = w.at(L.tmp), tmp2 = w.at(L.tmp2), k = w.at(L.k),
      ystage = w.at(L.ystage), ghimj = w.at(L.ghimj), jac = w.at(L.jac), djdt = w.at(L.djdt),
      hes = w.at(L.hes), u = w.at(L.u), v = w.at(L.v);
  const int S = tab.S;
  const long SN = 6L * NVAR;  // one adjoint's stage block in U and V
  const int direction = (tend >= tstart) ? 1 : -1;
  for (int sp = npush - 1; sp > 0; sp--) {
    // ros_DPop
    Col e = w.at(L.traj + (long)sp * L.entry);
    const double h = e[0];
    const double t = e[1];
    for (int i = 0; i < NVAR * S; i++) {
      ystage[i] = e[2 + i];
      k[i] = e[2 + 6L * NVAR + i];
    }
    if (c.save_lu) {
      for (int i = 0; i < LU_NZ; i++) ghimj[i] = e[2 + 12L * NVAR + i];
    } else {
      adj_rates(env, t, y, rconst);
      Jac_SP(ystage, env.fix, rconst, ghimj);
      st.njac++;
      const double tau = 1.0 / (direction * h * tab.Gamma[0]);
      wscal(LU_NZ, -1.0, ghimj);
      for (int i = 0; i < NVAR; i++) ghimj[LU_DIAG[i]] = ghimj[LU_DIAG[i]] + tau;
      (void)KppDecomp(ghimj);
      st.ndec++;
    }
    adj_rates(env, t, y, rconst);
    Hessian(ystage, env.fix, rconst, hes);
    for (int is = S - 1; is >= 0; is--) {
      const long istart = (long)NVAR * is;
      for (int m = 0; m < nadj; m++) {
        Col um = u.at(m * SN + istart);
        wcopy(NVAR, lambda.at((long)m * NVAR), um);
        wscal(NVAR, tab.M[is], um);
      }
      for (int j = is + 1; j < S; j++) {
        const long jstart = (long)NVAR * j;
        const double ha = tab.A[j * (j - 1) / 2 + is];
        const double hc = tab.C[j * (j - 1) / 2 + is] / (direction * h);
        for (int m = 0; m < nadj; m++) {
          Col um = u.at(m * SN + istart);
          waxpy(NVAR, ha, v.at(m * SN + jstart), um);
          waxpy(NVAR, hc, u.at(m * SN + jstart), um);
        }
      }
      for (int m = 0; m < nadj; m++) {
        Col um = u.at(m * SN + istart);
        KppSolveTR(ghimj, um, um);
        st.nsol++;
      }
      const double tau = t + tab.Alpha[is] * direction * h;
      adj_rates(env, tau, y, rconst);
      Col yst = ystage.at(istart);
      Jac_SP(yst, env.fix, rconst, jac);
      st.njac++;
      for (int m = 0; m < nadj; m++) {
        Col um = u.at(m * SN + istart), vm = v.at(m * SN + istart);
        JacTR_SP_Vec(jac, um, vm);
      }
    }
    if (!c.autonomous) {
      // ros_JacTimeDerivative (:1791-1811) at the step's start; Jac is the
      // last one evaluated, the first stage's
      const double delta = KPP_POW(kRoundoff, 0.5) * ros_max(kAdjDeltaMin, ros_abs(t));
      adj_rates(env, t + delta, y, rconst);
      Jac_SP(ystage, env.fix, rconst, djdt);
      st.njac++;
      waxpy(LU_NZ, -1.0, jac, djdt);
      wscal(LU_NZ, 1.0 / delta, djdt);
    }
    for (int is = 0; is < S; is++) {
      const long istart = (long)NVAR * is;
      for (int m = 0; m < nadj; m++) {
        Col lm = lambda.at((long)m * NVAR);
        waxpy(NVAR, 1.0, v.at(m * SN + istart), lm);
        Col um = u.at(m * SN + istart), ki = k.at(istart);
        HessTR_Vec(hes, um, ki, tmp);
        waxpy(NVAR, 1.0, tmp, lm);
      }
    }
    if (!c.autonomous) {
      for (int m = 0; m < nadj; m++) {
        for (int i = 0; i < NVAR; i++) tmp[i] = 0.0;
        for (int is = 0; is < S; is++) waxpy(NVAR, tab.Gamma[is], u.at(m * SN + (long)NVAR * is), tmp);
        JacTR_SP_Vec(djdt, tmp, tmp2);
        Col lm = lambda.at((long)m * NVAR);
        waxpy(NVAR, h, tmp2, lm);
      }
    }
  }
  return 1;
}

// RosenbrockADJ (:191-597) for one cell: controls, forward pass, backward
// pass.  y (VAR) and lambda in place; returns IERR.
__device__ inline int rosenbrock_adj_cell(const CellEnv& env, const int* icntrl,
                                          const double* rcntrl, const double* atol,
                                          const double* rtol, double tstart, double tend,
                                          Col y, Col lambda, int nadj, int bufsize, Col w,
                                          AdjStatus& st) {
  st = AdjStatus{0, 0, 0, 0, 0, 0, 0, 0, 0.0, 0.0, 0.0};
  AdjControls c;
  const int bad = adj_controls(icntrl, rcntrl, atol, rtol, bufsize, tstart, tend, c);
  if (bad) return bad;
  const AdjTableau tab = adj_tableau(c.method);
  const AdjLayout L = adj_layout(nadj, bufsize, c.save_lu);
  int npush = 0;
  const int ierr = adj_forward(env, c, tab, atol, rtol, tstart, tend, y, w, L, npush, st);
  if (ierr < 0) return ierr;
  if (!c.discrete) return ierr;
  return adj_backward(env, c, tab, tstart, tend, y, lambda, nadj, w, L, npush, st);
}

}  // namespace kpp_adj
