// Warp-cooperative Rosenbrock kernel: one warp integrates one cell whose whole
// work set (state vectors, stage vectors, LU matrix, rate constants and the
// Fun/Jacobian temporaries; ~19 KB for saprc99) lives in shared memory, so the
// time loop never touches HBM.  Included by kpp_rosenbrock.cu in the parts
// that instantiate one Rosenbrock method.
//
// Bit-identical to the thread-per-cell kernel (and so to the reference's
// arithmetic): the 32 lanes only run computations that are independent of
// each other, and every value is produced by the same operation sequence as
// the unrolled device functions (kppcu's kpp_warp schedules):
//   Fun     equation rates A[j] in parallel; each Vdot row summed by one lane
//           in equation order
//   Jac     partial derivatives B in parallel; each matrix entry summed by one
//           lane in equation order, negated, diagonal shifted by 1/(h*gamma)
//   LU      right-looking by pivot; an element receives its updates in
//           increasing pivot order, the order of util/sutil.c's row loop
//   solves  forward by pivot (a row's terms in increasing column order);
//           backward by dependency level, one lane per row
//   norm    squared scaled errors in parallel, summed in species order
// The scalar control (step size, accept/reject, counters) is computed by all
// lanes redundantly from identical values, so every branch is warp-uniform.
#pragma once

namespace warpk {

namespace W = kpp_warp;

constexpr int kAB = NREACT > W::NB ? NREACT : W::NB;
constexpr int kWarpStages = 6;

// Shared-memory layout of one cell (offsets in doubles).
template <int S>
struct Layout {
  static constexpr int Y = 0, YNEW = NVAR, FCN0 = 2 * NVAR, FCN = 3 * NVAR, DFDT = 4 * NVAR,
                       YERR = 5 * NVAR, K = 6 * NVAR, JVS = K + S * NVAR, RC = JVS + LU_NZ,
                       AB = RC + NREACT, EX = AB + kAB, TOTAL = EX + NFIX + 1;
};

// Product operand: variable species, fixed species, or the padding 1.0.
__device__ __forceinline__ double operand(const double* V, const double* ex, int idx) {
  return idx < NVAR ? V[idx] : ex[idx - NVAR];
}

// Vdot = f(V) with rate constants rc; A is the equation-rate temporary.
__device__ __forceinline__ void fun(const double* V, const double* ex, const double* rc, double* A,
                                    double* out, int lane) {
  for (int t = lane; t < W::NA; t += 32) {
    double v = W::a_rct[t] >= 0 ? rc[W::a_rct[t]] : W::a_k1[t];
    if (W::a_k2[t] != 1.0) v = v * W::a_k2[t];
#pragma unroll
    for (int f = 0; f < W::MAXF; f++) {
      const int idx = W::a_f[t * W::MAXF + f];
      if (idx != W::KPP_WOPND_ONE) v = v * operand(V, ex, idx);
    }
    A[W::a_eq[t]] = v;
  }
  __syncwarp();
  for (int i = lane; i < NVAR; i += 32) {
    const int b = W::v_ptr[i], e = W::v_ptr[i + 1];
    double acc = 0.0;
    if (b < e) {
      acc = W::v_c[b] * A[W::v_j[b]];
      for (int k = b + 1; k < e; k++) acc = acc + W::v_c[k] * A[W::v_j[k]];
    }
    out[i] = acc;
  }
  __syncwarp();
}

// J = -Jac(V) + ghinv I in the LU pattern; B is the derivative temporary.
__device__ __forceinline__ void jac_matrix(const double* V, const double* ex, const double* rc,
                                           double* B, double* J, double ghinv, int lane) {
  for (int t = lane; t < W::NB; t += 32) {
    double v = W::b_rct[t] >= 0 ? rc[W::b_rct[t]] : W::b_k1[t];
    if (W::b_k2[t] != 1.0) v = v * W::b_k2[t];
#pragma unroll
    for (int f = 0; f < W::MAXF; f++) {
      const int idx = W::b_f[t * W::MAXF + f];
      if (idx != W::KPP_WOPND_ONE) v = v * operand(V, ex, idx);
    }
    B[t] = v;
  }
  __syncwarp();
  for (int n = lane; n < LU_NZ; n += 32) {
    const int b = W::j_ptr[n], e = W::j_ptr[n + 1];
    double acc = 0.0;
    if (b < e) {
      acc = W::j_c[b] * B[W::j_b[b]];
      for (int k = b + 1; k < e; k++) acc = acc + W::j_c[k] * B[W::j_b[k]];
    }
    J[n] = -acc;
  }
  __syncwarp();
  for (int i = lane; i < NVAR; i += 32) J[W::lu_diag[i]] = J[W::lu_diag[i]] + ghinv;
  __syncwarp();
}

__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    int w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// In-place no-pivot sparse LU; returns k+1 for the first row whose diagonal
// is zero on entry to its elimination (it is the original value: a row is
// only changed by its own elimination), 0 on success.
__device__ __forceinline__ int decomp(double* J, int lane) {
  int bad = NVAR;
  for (int i = lane; i < NVAR; i += 32)
    if (J[W::lu_diag[i]] == 0.0 && i < bad) bad = i;
  bad = warp_min(bad);
  if (bad < NVAR) return bad + 1;
  for (int p = 0; p < W::NPIV; p++) {
    const double d = J[W::lu_diag[W::lu_piv[p]]];
    for (int t = W::lu_lptr[p] + lane; t < W::lu_lptr[p + 1]; t += 32) {
      const int q = W::lu_l[t];
      const double a = -J[q] / d;
      J[q] = -a;
    }
    __syncwarp();
    for (int t = W::lu_uptr[p] + lane; t < W::lu_uptr[p + 1]; t += 32)
      J[W::lu_ut[t]] = J[W::lu_ut[t]] + (-J[W::lu_um[t]]) * J[W::lu_us[t]];
    __syncwarp();
  }
  return 0;
}

// Solve (LU) x = b in place.
__device__ __forceinline__ void solve(const double* J, double* X, int lane) {
  for (int p = 0; p < W::NFWP; p++) {
    const double xj = X[W::fw_piv[p]];
    for (int t = W::fw_ptr[p] + lane; t < W::fw_ptr[p + 1]; t += 32) {
      const int i = W::fw_row[t];
      X[i] = X[i] - J[W::fw_pos[t]] * xj;
    }
    __syncwarp();
  }
  for (int lv = 0; lv < W::NLEV; lv++) {
    for (int t = W::bw_lptr[lv] + lane; t < W::bw_lptr[lv + 1]; t += 32) {
      const int i = W::bw_rows[t];
      double s = X[i];
      for (int jj = W::lu_diag[i] + 1; jj < W::lu_crow[i + 1]; jj++) s = s - J[jj] * X[W::lu_icol[jj]];
      X[i] = s / J[W::lu_diag[i]];
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void vaxpy(double alpha, const double* x, double* y, int lane) {
  if (alpha == 0.0) return;  // WAXPY's early return (util/blas.c:64), warp-uniform
  for (int i = lane; i < NVAR; i += 32) y[i] = y[i] + alpha * x[i];
  __syncwarp();
}

__device__ __forceinline__ void vcopy(const double* x, double* y, int lane) {
  for (int i = lane; i < NVAR; i += 32) y[i] = x[i];
  __syncwarp();
}

// The rate constants that change with the evaluation time (SUN from
// Update_SUN(t), or rates depending on TIME or the state), recomputed by lane 0.
__device__ __forceinline__ void rates_at(const CellEnv& env, double t, double* rc, const double* y,
                                         const double* ex, int lane) {
  if (lane == 0) {
    if (KPP_RATES_SUN > 0 && env.sun_fixed < 0.0)
      kpp_rconst_sun(rc, t, env.temp, env.cfactor, kpp_update_sun(t), y, ex);
    if (KPP_RATES_DYNAMIC > 0)
      kpp_rconst_dynamic(rc, t, env.temp, env.cfactor, cell_sun(env, t), y, ex);
  }
  __syncwarp();
}

// RosenbrockIntegrator (int/rosenbrock.c:450-627) for the cell in `sm`.
template <int METHOD>
__device__ int integrate(const CellEnv& env, double* sm, int lane, double tstart, double tend,
                         const double* atol, const double* rtol, bool autonomous, bool vectortol,
                         int max_no_steps, double hmin, double hmax, double hstart, double facmin,
                         double facmax, double facrej, double facsafe, double& texit,
                         double& hexit, Stats& st) {
  constexpr Tableau tab = make_tableau(METHOD);
  constexpr int S = tab.S;
  using L = Layout<kWarpStages>;
  double* y = sm + L::Y;
  double* ynew = sm + L::YNEW;
  double* fcn0 = sm + L::FCN0;
  double* fcn = sm + L::FCN;
  double* dfdt = sm + L::DFDT;
  double* yerr = sm + L::YERR;
  double* jvs = sm + L::JVS;
  double* rc = sm + L::RC;
  double* ab = sm + L::AB;
  double* ex = sm + L::EX;
  auto kst = [&](int s) { return sm + L::K + s * NVAR; };

  const bool varying = KPP_RATES_DYNAMIC > 0 || (KPP_RATES_SUN > 0 && env.sun_fixed < 0.0);
  double t = tstart;
  hexit = 0.0;
  double h = ros_min(hstart, hmax);
  if (ros_abs(h) <= 10.0 * kRoundoff) h = kDeltaMin;
  const int direction = (tend >= tstart) ? +1 : -1;
  bool reject_last = false, reject_more = false;

  while (((direction > 0) && ((t - tend) + kRoundoff <= 0.0)) ||
         ((direction < 0) && ((tend - t) + kRoundoff <= 0.0))) {
    if (st.nstp > max_no_steps) { texit = t; return KPP_B200_IERR_TOO_MANY_STEPS; }
    if (((t + 0.1 * h) == t) || (h <= kRoundoff)) { texit = t; return KPP_B200_IERR_STEP_TOO_SMALL; }
    hexit = h;
    h = ros_min(h, ros_abs_diff(tend, t));

    if (varying) rates_at(env, t, rc, y, ex, lane);
    fun(y, ex, rc, ab, fcn0, lane);
    st.nfun++;
    if (!autonomous) {
      double delta = sqrt(kRoundoff) * ros_max(kDeltaMin, ros_abs(t));
      if (varying) {
        rates_at(env, t + delta, rc, y, ex, lane);
        fun(y, ex, rc, ab, dfdt, lane);
        rates_at(env, t, rc, y, ex, lane);
      } else {
        vcopy(fcn0, dfdt, lane);  // Fun(T+Delta) would see the same rates and state
      }
      st.nfun++;
      vaxpy(-1.0, fcn0, dfdt, lane);
      const double inv = 1.0 / delta;
      if (inv != 1.0) {
        for (int i = lane; i < NVAR; i += 32) dfdt[i] = inv * dfdt[i];
        __syncwarp();
      }
    }
    st.njac++;

    bool retry = false;
    for (;;) {
      if (retry && varying) rates_at(env, t, rc, y, ex, lane);
      retry = true;
      // ros_PrepareMatrix (int/rosenbrock.c:686-737)
      {
        int nconsecutive = 0;
        bool singular = false;
        for (;;) {
          const double ghinv = 1.0 / (direction * h * tab.Gamma[0]);
          jac_matrix(y, ex, rc, ab, jvs, ghinv, lane);
          const int ising = decomp(jvs, lane);
          st.ndec++;
          if (ising == 0) break;
          st.nsng++;
          nconsecutive++;
          if (nconsecutive <= 5) {
            h = h * 0.5;
          } else {
            singular = true;
            break;
          }
        }
        if (singular) { texit = t; return KPP_B200_IERR_SINGULAR; }
      }
#pragma unroll
      for (int s = 0; s < S; s++) {
        if (s == 0) {
          vcopy(fcn0, fcn, lane);
        } else if (tab.NewF[s]) {
          vcopy(y, ynew, lane);
#pragma unroll
          for (int j = 0; j < s; j++) vaxpy(tab.A[s * (s - 1) / 2 + j], kst(j), ynew, lane);
          const double tau = t + tab.Alpha[s] * direction * h;
          if (varying) rates_at(env, tau, rc, y, ex, lane);
          fun(ynew, ex, rc, ab, fcn, lane);
          st.nfun++;
        }
        vcopy(fcn, kst(s), lane);
#pragma unroll
        for (int j = 0; j < s; j++) {
          const double hc = tab.C[s * (s - 1) / 2 + j] / (direction * h);
          vaxpy(hc, kst(j), kst(s), lane);
        }
        if ((!autonomous) && (tab.Gamma[s] != 0.0)) {
          const double hg = direction * h * tab.Gamma[s];
          vaxpy(hg, dfdt, kst(s), lane);
        }
        solve(jvs, kst(s), lane);
        st.nsol++;
      }

      vcopy(y, ynew, lane);
#pragma unroll
      for (int j = 0; j < S; j++) vaxpy(tab.M[j], kst(j), ynew, lane);
      for (int i = lane; i < NVAR; i += 32) yerr[i] = 0.0;
      __syncwarp();
#pragma unroll
      for (int j = 0; j < S; j++) vaxpy(tab.E[j], kst(j), yerr, lane);
      // ros_ErrorNorm: terms in parallel (into fcn, free until the next
      // step), summed in species order by every lane
      {
        const double a0 = atol[0], r0 = rtol[0];
        for (int i = lane; i < NVAR; i += 32) {
          const double ymax = ros_max(ros_abs(y[i]), ros_abs(ynew[i]));
          const double scale = vectortol ? (atol[i] + rtol[i] * ymax) : (a0 + r0 * ymax);
          fcn[i] = (yerr[i] * yerr[i]) / (scale * scale);
        }
        __syncwarp();
      }
      double err = 0.0;
      for (int i = 0; i < NVAR; i++) err = err + fcn[i];
      err = sqrt(err / (double)NVAR);
      __syncwarp();

      const double fac = ros_min(facmax, ros_max(facmin, facsafe / pow(err, 1.0 / tab.ELO)));
      double hnew = h * fac;

      st.nstp++;
      if ((err <= 1.0) || (h <= hmin)) {
        st.nacc++;
        vcopy(ynew, y, lane);
        t += direction * h;
        hnew = ros_max(hmin, ros_min(hnew, hmax));
        if (reject_last) hnew = ros_min(hnew, h);
        reject_last = false;
        reject_more = false;
        h = hnew;
        break;
      } else {
        if (st.nacc >= 1) st.nrej++;
        if (reject_more) hnew = h * facrej;
        reject_more = reject_last;
        reject_last = true;
        h = hnew;
      }
    }
  }
  texit = t;
  return KPP_B200_IERR_SUCCESS;
}

// Rosenbrock (int/rosenbrock.c:137-446) controls, as rosenbrock_cell.
template <int METHOD>
__device__ int rosenbrock(const CellEnv& env, double* sm, int lane, double tstart, double tend,
                          const double* atol, const double* rtol, const LaunchArgs& a,
                          double rpar2, Stats& st, double& texit, double& hexit) {
  const int* ipar = a.ipar;
  const double* rpar = a.rpar;
  const bool autonomous = !(ipar[0] == 0);
  const bool vectortol = (ipar[1] == 0);
  const int uplimtol = vectortol ? NVAR : 1;
  const int max_no_steps = (ipar[2] == 0) ? 100000 : ipar[2];
  if (max_no_steps < 0) return KPP_B200_IERR_MAXSTEPS_BAD;
  if ((ipar[3] < 1) || (ipar[3] > 5)) return KPP_B200_IERR_METHOD;
  const double hmin = rpar[0];
  if (rpar[0] < 0.0) return KPP_B200_IERR_HBOUNDS;
  const double hmax = (rpar[1] == 0.0) ? ros_abs_diff(tend, tstart)
                                       : ros_min(ros_abs(rpar[1]), ros_abs_diff(tend, tstart));
  if (rpar[1] < 0.0) return KPP_B200_IERR_HBOUNDS;
  const double hstart = (rpar2 == 0.0) ? ros_max(hmin, kDeltaMin)
                                       : ros_min(ros_abs(rpar2), ros_abs_diff(tend, tstart));
  if (rpar2 < 0.0) return KPP_B200_IERR_HBOUNDS;
  const double facmin = (rpar[3] == 0.0) ? 0.2 : rpar[3];
  if (rpar[3] < 0.0) return KPP_B200_IERR_FACTORS;
  const double facmax = (rpar[4] == 0.0) ? 6.0 : rpar[4];
  if (rpar[4] < 0.0) return KPP_B200_IERR_FACTORS;
  const double facrej = (rpar[5] == 0.0) ? 0.1 : rpar[5];
  if (rpar[5] < 0.0) return KPP_B200_IERR_FACTORS;
  const double facsafe = (rpar[6] == 0.0) ? 0.9 : rpar[6];
  if (rpar[6] < 0.0) return KPP_B200_IERR_FACTORS;
  for (int i = 0; i < uplimtol; i++)
    if ((atol[i] <= 0.0) || (rtol[i] <= 10.0 * kRoundoff) || (rtol[i] >= 1.0))
      return KPP_B200_IERR_TOLERANCES;
  return integrate<METHOD>(env, sm, lane, tstart, tend, atol, rtol, autonomous, vectortol,
                           max_no_steps, hmin, hmax, hstart, facmin, facmax, facrej, facsafe,
                           texit, hexit, st);
}

constexpr size_t kSmemBytes = sizeof(double) * (size_t)Layout<kWarpStages>::TOTAL;

// One warp (block) per cell, grid-stride over cells.  `rates` holds each
// cell's rate constants that are fixed for the call, [NREACT][rates_ld] with
// cell index fastest, written by the rate pre-pass.
template <int METHOD>
__global__ void __launch_bounds__(32) kernel(const LaunchArgs a, const double* __restrict__ rates,
                                             long rates_ld) {
  extern __shared__ double sm[];
  using L = Layout<kWarpStages>;
  const int lane = threadIdx.x;
  const long ld = a.ld;
  for (long c = blockIdx.x; c < a.ncells; c += gridDim.x) {
    const int cell = (int)c;
    CellEnv env;
    load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, cell);
    for (int i = lane; i < NVAR; i += 32) sm[L::Y + i] = a.var[i * ld + cell];
    for (int i = lane; i < NREACT; i += 32) sm[L::RC + i] = rates[i * rates_ld + c];
    if (lane == 0) {
      for (int i = 0; i < NFIX; i++) sm[L::EX + i] = env.fix[i];
      sm[L::EX + NFIX] = 1.0;
    }
    __syncwarp();

    Stats st = {0, 0, 0, 0, 0, 0, 0, 0};
    double texit = 0.0, hexit = 0.0;
    const double rpar2 = a.hstart ? a.hstart[cell] : a.rpar[2];
    const int ierr = rosenbrock<METHOD>(env, sm, lane, a.tstart[cell], a.tend[cell], a.atol,
                                        a.rtol, a, rpar2, st, texit, hexit);
    __syncwarp();
    for (int i = lane; i < NVAR; i += 32) a.var[i * ld + cell] = sm[L::Y + i];
    if (lane == 0) {
      a.ierr[cell] = ierr;
      const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
      for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] = sv[i];
      a.rstatus[cell] = texit;
      a.rstatus[ld + cell] = hexit;
    }
    __syncwarp();
  }
}

}  // namespace warpk
