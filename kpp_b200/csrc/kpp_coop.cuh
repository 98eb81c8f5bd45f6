// Warp-per-cell Rosenbrock kernel: one warp integrates one grid cell whose
// whole work set (state and stage vectors, the Rosenbrock matrix and its LU
// factors, the Fun/Jac products; 14.5 KB for saprc99 with Rodas3) lives in
// shared memory, so the time loop never touches HBM.  Included by
// kpp_rosenbrock.cu in the parts that instantiate one Rosenbrock method.
//
// Schedules.  kppcu spreads every phase over the warp's 32 lanes with static
// schedules (namespace kpp_coop of the mechanism header; see its emitter),
// which each CTA copies once into shared memory:
//   products   Fun's equation rates and Jac_SP's partial derivatives, one per
//              lane and round: weight (rate constant x stoichiometric factor,
//              held in registers for the whole cell) times the reactants
//   sums       each Vdot row / Jacobian entry summed by one lane in equation
//              order (lane streams of packed entries)
//   LU         the operations of util/sutil.c's loop list-scheduled into
//              iterations separated by warp barriers
//   forward    substitution: each row's left-to-right sum owned by one lane
//              and advanced as its operands become final
// The backward substitution is close to one dependent chain (the rows of the
// dense trailing block each begin with the row just below them), so one lane
// runs it as the mechanism header's straight-line kpp_solve_bw while the warp
// waits.  Spread over the lanes, every link of the chain paid table reads and
// a warp barrier, and the phase took half of the kernel's time; on one lane
// the kernel runs about twice as fast (saprc99, 2^17 cells).
// Only operations that do not depend on each other run side by side, and each
// value is produced by the operation sequence of the unrolled functions, so the
// kernel is bit-identical to the thread-per-cell kernel (and performs the
// reference's arithmetic: int/rosenbrock.c, util/sutil.c:2-23,
// src/gen.c:642-724, 1185-1322, 1960-2034).  The scalar control (step size,
// accept/reject, counters) runs redundantly in every lane on identical
// values, so every branch of the controller is warp-uniform.
//
// Rate constants must be fixed for the whole call (SUN given per cell, or no
// SUN-dependent rates, and no rates that depend on time or concentrations):
// lane 0 evaluates them once per cell and every lane derives its product
// weights from them.  Other mechanisms and inputs use the thread-per-cell
// kernel.
#pragma once

namespace coop {

namespace K = kpp_coop;

constexpr int kSmemMax = 227 * 1024;  // shared memory one CTA can hold on sm_100
constexpr unsigned kNop = 0xFFFFFFFFu;

// Shared memory of one cell (offsets in doubles), for an S-stage method.
template <int S>
struct Cell {
  static constexpr int V0 = 0;                  // y, FIX, 1.0 (the products' operands)
  static constexpr int FCN0 = V0 + K::NEXT;     // Fun(T, y)
  static constexpr int DFDT = FCN0 + NVAR;
  static constexpr int JVS = DFDT + NVAR;       // Rosenbrock matrix / LU factors
  static constexpr int A = JVS + LU_NZ;         // Fun's equation rates
  static constexpr int V1 = A + K::NA;          // ynew, FIX, 1.0
  static constexpr int FCN = V1 + K::NEXT;      // stage Fun; then Yerr and the error terms
  static constexpr int KS = FCN + NVAR;         // stage vectors
  static constexpr int END = KS + S * NVAR;
  // Jac_SP's partial derivatives reuse [FCN, END) (dead while the matrix is
  // built) when they fit there
  static constexpr int B = (END - FCN >= K::NB) ? FCN : END;
  static constexpr int TOTAL = (B == FCN) ? END : END + K::NB;
  static_assert(LU_NZ + K::NA >= NREACT, "rate constants are staged in [JVS, V1)");
};

constexpr size_t kTabBytes = ((size_t)K::TAB_WORDS * 4 + 15) / 16 * 16;
constexpr size_t kTablesBytes = kTabBytes + (size_t)K::NKC * 8;

// Warps (cells) of a CTA: as many cells as shared memory holds beside the
// tables, at most kMaxWarps.  For mechanisms of saprc99's size the phases'
// staged operands need about 168 registers per thread, which 12 warps of 32
// threads allow (at 13 warps ptxas caps the kernel at 128 registers and it
// spills 2.4 KB per thread); small mechanisms take up to 32 cells.
constexpr int kMaxWarps = LU_NZ > 256 ? 12 : 32;
template <int S>
constexpr int warps_per_cta() {
  const long w = ((long)kSmemMax - (long)kTablesBytes) / ((long)Cell<S>::TOTAL * 8);
  return w > kMaxWarps ? kMaxWarps : (w < 1 ? 0 : (int)w);
}

template <int S>
constexpr size_t smem_bytes() {
  return kTablesBytes + (size_t)warps_per_cta<S>() * Cell<S>::TOTAL * 8;
}

// ---- phases (all lanes of the warp call each one) ----------------------------

// Every phase below first loads what its lanes need -- table entries, then
// their operands -- into registers and only then computes, so that each
// lane's loads overlap instead of forming one long chain of dependent
// shared-memory round trips.  Within one iteration of a schedule no lane reads
// what another lane of that iteration writes, and a lane's own entries of one
// iteration do not depend on each other, so all loads of an iteration can go
// first.

// Product weights of a lane: round r covers product r*32 + lane.
template <int R>
__device__ __forceinline__ void weights(const unsigned* __restrict__ tab, int off,
                                        const double* __restrict__ kc,
                                        const double* __restrict__ rc, double (&w)[R], int lane) {
  constexpr unsigned RM = (1u << K::RATE_BITS) - 1;
#pragma unroll
  for (int r = 0; r < R; r++) {
    const unsigned e = tab[off + r * 32 + lane];
    const unsigned rct = e & RM;
    const double base = (rct != (unsigned)K::NO_RATE) ? rc[rct] : kc[(e >> K::RATE_BITS) & 4095];
    w[r] = base * kc[(e >> (K::RATE_BITS + 12)) & 4095];
  }
}

// out[t] = weight(t) x the reactant factors of product t, for t < N.  The
// table is padded to whole rounds with the constant 1.0 as every factor.
template <int R, int N>
__device__ __forceinline__ void products(const unsigned* __restrict__ tab, int off,
                                         const double (&w)[R], const double* __restrict__ vext,
                                         double* __restrict__ out, int lane) {
  unsigned f[R];
#pragma unroll
  for (int r = 0; r < R; r++) f[r] = tab[off + r * 32 + lane];
  double v[R][K::MAXF];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int k = 0; k < K::MAXF; k++) v[r][k] = vext[(f[r] >> (8 * k)) & 255u];
#pragma unroll
  for (int r = 0; r < R; r++) {
    double x = w[r];
#pragma unroll
    for (int k = 0; k < K::MAXF; k++) x = x * v[r][k];
    if (r * 32 + lane < N) out[r * 32 + lane] = x;
  }
}

// The lane streams of a sum phase: out[dst] = sum of kc[coef] * src[idx] in
// order, negated for the Rosenbrock matrix (NEG), with 1/(h gamma) added on
// diagonal entries (DIAG).  Entries are taken in chunks of CH: their table
// words, then their operands, then the running sums.
template <int L, bool NEG, bool DIAG>
__device__ __forceinline__ void sums(const unsigned* __restrict__ tab, int off,
                                     const double* __restrict__ kc,
                                     const double* __restrict__ src, double* __restrict__ out,
                                     double ghinv, int lane) {
  constexpr int SB = K::SUM_SRC_BITS, CB = K::SUM_COEF_BITS, FB = SB + CB;
  constexpr unsigned SM = (1u << SB) - 1, CM = (1u << CB) - 1;
  constexpr int CH = 8;
  double acc = 0.0;
#pragma unroll 2
  for (int k0 = 0; k0 < L; k0 += CH) {
    unsigned e[CH];
    double p[CH];
#pragma unroll
    for (int j = 0; j < CH; j++) e[j] = (k0 + j < L) ? tab[off + (k0 + j) * 32 + lane] : kNop;
#pragma unroll
    for (int j = 0; j < CH; j++) {
      const unsigned ej = (e[j] == kNop) ? 0u : e[j];  // a NOP reads entry 0's operands
      p[j] = kc[(ej >> SB) & CM] * src[ej & SM];
    }
#pragma unroll
    for (int j = 0; j < CH; j++) {
      const unsigned ej = e[j];
      if (ej == kNop) continue;
      double val;
      if ((ej >> (FB + 2)) & 1u) {
        val = NEG ? -0.0 : 0.0;
      } else {
        acc = ((ej >> FB) & 1u) ? p[j] : acc + p[j];
        val = NEG ? -acc : acc;
      }
      if ((ej >> (FB + 1)) & 1u) {
        if (DIAG && ((ej >> (FB + 3)) & 1u)) val = val + ghinv;
        out[ej >> (FB + 4)] = val;
      }
    }
  }
}

__device__ __forceinline__ int lane_count(const unsigned* __restrict__ tab, int off, int it,
                                          int lane) {
  return (tab[off + it * 4 + (lane >> 3)] >> ((lane & 7) * 4)) & 15u;
}

// Vdot = f(vext) (Fun, aggregate form).
template <int S>
__device__ __forceinline__ void fun(const unsigned* tab, const double* kc,
                                    const double (&wf)[K::RF], const double* vext, double* sm,
                                    double* out, int lane) {
  products<K::RF, K::NA>(tab, K::O_PF, wf, vext, sm + Cell<S>::A, lane);
  __syncwarp();
  sums<K::LV, false, false>(tab, K::O_SV, kc, sm + Cell<S>::A, out, 0.0, lane);
  __syncwarp();
}

// JVS = -Jac_SP(y) + ghinv I.
template <int S>
__device__ __forceinline__ void jac_matrix(const unsigned* tab, const double* kc,
                                           const double (&wj)[K::RJ], double* sm, double ghinv,
                                           int lane) {
  products<K::RJ, K::NB>(tab, K::O_PJ, wj, sm + Cell<S>::V0, sm + Cell<S>::B, lane);
  __syncwarp();
  sums<K::LJ, true, true>(tab, K::O_SJ, kc, sm + Cell<S>::B, sm + Cell<S>::JVS, ghinv, lane);
  __syncwarp();
}

__device__ __forceinline__ int warp_min(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// In-place no-pivot sparse LU; returns k+1 for the first row whose diagonal
// is zero on entry to its elimination (its original value: util/sutil.c only
// changes a row during that row's own elimination), 0 on success.
__device__ __forceinline__ int decomp(const unsigned* __restrict__ tab, double* J, int lane) {
  int bad = NVAR;
  for (int i = lane; i < NVAR; i += 32)
    if (J[tab[K::O_DIAG + i]] == 0.0 && i < bad) bad = i;
  bad = warp_min(bad);
  if (bad < NVAR) return bad + 1;
  constexpr int B = K::LU_BITS, CAP = K::LU_CAP;
  constexpr unsigned M = (1u << B) - 1;
  int pos = 0;
  int n = lane_count(tab, K::O_CLU, 0, lane);
  for (int it = 0; it < K::IT_LU; it++) {
    unsigned e[CAP];
    double vt[CAP], vm[CAP], vs[CAP];
#pragma unroll
    for (int j = 0; j < CAP; j++) e[j] = (j < n) ? tab[K::O_LU + (pos + j) * 32 + lane] : 0u;
#pragma unroll
    for (int j = 0; j < CAP; j++) {
      vt[j] = J[(e[j] >> (2 * B)) & M];
      vm[j] = J[(e[j] >> B) & M];
      vs[j] = J[e[j] & M];
    }
    const int n_next = (it + 1 < K::IT_LU) ? lane_count(tab, K::O_CLU, it + 1, lane) : 0;
#pragma unroll
    for (int j = 0; j < CAP; j++)
      if (j < n) J[(e[j] >> (2 * B)) & M] = (e[j] >> 31) ? vt[j] / vs[j] : vt[j] + (-vm[j]) * vs[j];
    pos += n;
    n = n_next;
    __syncwarp();
  }
  return 0;
}

// Forward substitution in place (unit lower triangle, KppSolve's first loop).
__device__ __forceinline__ void forward(const unsigned* __restrict__ tab, const double* J,
                                        double* X, int lane) {
  constexpr int B = K::LU_BITS, C = K::X_BITS, F = B + 2 * C, CAP = K::SOLVE_CAP;
  double acc = 0.0;
  int pos = 0;
  int n = lane_count(tab, K::O_CFW, 0, lane);
  for (int it = 0; it < K::IT_FW; it++) {
    unsigned e[CAP];
    double jv[CAP], xv[CAP], xs[CAP];
#pragma unroll
    for (int j = 0; j < CAP; j++) e[j] = (j < n) ? tab[K::O_FW + (pos + j) * 32 + lane] : 0u;
#pragma unroll
    for (int j = 0; j < CAP; j++) {
      jv[j] = J[e[j] & ((1u << B) - 1)];
      xv[j] = X[(e[j] >> B) & ((1u << C) - 1)];
      xs[j] = X[(e[j] >> (B + C)) & ((1u << C) - 1)];
    }
    const int n_next = (it + 1 < K::IT_FW) ? lane_count(tab, K::O_CFW, it + 1, lane) : 0;
    // the running sums
#pragma unroll
    for (int j = 0; j < CAP; j++) {
      if (j < n) {
        if ((e[j] >> F) & 1u) acc = xs[j];
        acc = acc - jv[j] * xv[j];
        if ((e[j] >> (F + 1)) & 1u) X[(e[j] >> (B + C)) & ((1u << C) - 1)] = acc;
      }
    }
    pos += n;
    n = n_next;
    __syncwarp();
  }
}

// The backward substitution on one lane, kept out of line: one copy of its
// straight-line code (about 2.5k instructions for saprc99) instead of one per
// unrolled stage, which relieves the instruction cache (9 % faster at 2^20
// cells).
static __device__ __noinline__ void solve_bw_lane(const double* J, double* X) {
  kpp_solve_bw(J, X);
}

// Solve (LU) x = b in place, b given in X: the forward substitution over the
// warp, the backward one on lane 0.
__device__ __forceinline__ void solve(const unsigned* __restrict__ tab, const double* J, double* X,
                                      int lane) {
  forward(tab, J, X, lane);
  if (lane == 0) solve_bw_lane(J, X);
  __syncwarp();
}

// ---- vector operations of the integrator (util/blas.c), lane-strided -------
__device__ __forceinline__ void vaxpy(double alpha, const double* x, double* y, int lane) {
  if (alpha == 0.0) return;  // WAXPY's early return (util/blas.c:64), warp-uniform
  for (int i = lane; i < NVAR; i += 32) y[i] = y[i] + alpha * x[i];
  __syncwarp();
}

__device__ __forceinline__ void vcopy(const double* x, double* y, int lane) {
  for (int i = lane; i < NVAR; i += 32) y[i] = x[i];
  __syncwarp();
}

// ---- RosenbrockIntegrator (int/rosenbrock.c:450-627) for the cell in `sm` ----
struct Weights {
  double f[K::RF], j[K::RJ];
};

template <int METHOD>
__device__ int integrate(const unsigned* tab, const double* kc, const Weights& w, double* sm,
                         int lane, double tstart, double tend, const double* atol,
                         const double* rtol, bool autonomous, bool vectortol, int max_no_steps,
                         double hmin, double hmax, double hstart, double facmin, double facmax,
                         double facrej, double facsafe, double& texit, double& hexit, Stats& st) {
  constexpr Tableau tab_m = make_tableau(METHOD);
  constexpr int S = tab_m.S;
  using L = Cell<S>;
  double* y = sm + L::V0;
  double* ynew = sm + L::V1;
  double* fcn0 = sm + L::FCN0;
  double* fcn = sm + L::FCN;
  double* dfdt = sm + L::DFDT;
  double* yerr = sm + L::FCN;  // after the stages: Yerr, then the error terms
  double* jvs = sm + L::JVS;
  auto kst = [&](int s) { return sm + L::KS + s * NVAR; };

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

    fun<S>(tab, kc, w.f, y, sm, fcn0, lane);  // FunTemplate(T, Y, Fcn0)
    st.nfun++;
    if (!autonomous) {
      // ros_FunTimeDerivative (:663-682); the rates are fixed over the call,
      // so Fun(T + Delta) equals Fcn0
      const double delta = sqrt(kRoundoff) * ros_max(kDeltaMin, ros_abs(t));
      vcopy(fcn0, dfdt, lane);
      st.nfun++;
      vaxpy(-1.0, fcn0, dfdt, lane);
      const double inv = 1.0 / delta;
      if (inv != 1.0) {
        for (int i = lane; i < NVAR; i += 32) dfdt[i] = inv * dfdt[i];
        __syncwarp();
      }
    }
    st.njac++;  // JacTemplate(T, Y, Jac0), evaluated with the matrix below

    for (;;) {  // until the step is accepted
      // ros_PrepareMatrix (:686-737): Ghimj = -Jac0 + 1/(H*gamma) I, LU;
      // the matrix is evaluated anew from the same inputs on every attempt
      {
        int nconsecutive = 0;
        bool singular = false;
        for (;;) {
          const double ghinv = 1.0 / (direction * h * tab_m.Gamma[0]);
          jac_matrix<S>(tab, kc, w.j, sm, ghinv, lane);
          const int ising = decomp(tab, jvs, lane);
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
        } else if (tab_m.NewF[s]) {
          vcopy(y, ynew, lane);
#pragma unroll
          for (int j = 0; j < s; j++) vaxpy(tab_m.A[s * (s - 1) / 2 + j], kst(j), ynew, lane);
          fun<S>(tab, kc, w.f, ynew, sm, fcn, lane);
          st.nfun++;
        }
        vcopy(fcn, kst(s), lane);
#pragma unroll
        for (int j = 0; j < s; j++) {
          const double hc = tab_m.C[s * (s - 1) / 2 + j] / (direction * h);
          vaxpy(hc, kst(j), kst(s), lane);
        }
        if ((!autonomous) && (tab_m.Gamma[s] != 0.0)) {
          const double hg = direction * h * tab_m.Gamma[s];
          vaxpy(hg, dfdt, kst(s), lane);
        }
        solve(tab, jvs, kst(s), lane);
        st.nsol++;
      }

      vcopy(y, ynew, lane);
#pragma unroll
      for (int j = 0; j < S; j++) vaxpy(tab_m.M[j], kst(j), ynew, lane);
      for (int i = lane; i < NVAR; i += 32) yerr[i] = 0.0;
      __syncwarp();
#pragma unroll
      for (int j = 0; j < S; j++) vaxpy(tab_m.E[j], kst(j), yerr, lane);
      // ros_ErrorNorm (:632-659): the terms in parallel (over Yerr, each lane
      // its own species), summed in species order by every lane
      {
        const double a0 = atol[0], r0 = rtol[0];
        for (int i = lane; i < NVAR; i += 32) {
          const double ymax = ros_max(ros_abs(y[i]), ros_abs(ynew[i]));
          const double scale = vectortol ? (atol[i] + rtol[i] * ymax) : (a0 + r0 * ymax);
          yerr[i] = (yerr[i] * yerr[i]) / (scale * scale);
        }
        __syncwarp();
      }
      double err = 0.0;
      for (int i = 0; i < NVAR; i++) err = err + yerr[i];
      err = sqrt(err / (double)NVAR);
      __syncwarp();

      const double fac =
          ros_min(facmax, ros_max(facmin, facsafe / KPP_POW(err, 1.0 / tab_m.ELO)));
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

// Rosenbrock (int/rosenbrock.c:137-446): validation and defaults, then the
// integrator, as rosenbrock_cell of the thread-per-cell kernel.
template <int METHOD>
__device__ int rosenbrock(const unsigned* tab, const double* kc, const Weights& w, double* sm,
                          int lane, double tstart, double tend, const LaunchArgs& a, double rpar2,
                          Stats& st, double& texit, double& hexit) {
  const int* ipar = a.ipar;
  const double* rpar = a.rpar;
  const double* atol = a.atol;
  const double* rtol = a.rtol;
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
  return integrate<METHOD>(tab, kc, w, sm, lane, tstart, tend, atol, rtol, autonomous, vectortol,
                           max_no_steps, hmin, hmax, hstart, facmin, facmax, facrej, facsafe,
                           texit, hexit, st);
}

// One cell: its state, rate constants and product weights, then one
// Rosenbrock call over [tstart, tend] or, with a.nchain >= 1, the driver loop
// around INTEGRATE (drv/general.c:59-76, int/rosenbrock.c:94-133): a.nchain
// calls of a.chain_dt seconds, each warm-started from the previous call's
// Hexit, counters summed, Texit/Hexit of the last call, IERR of the first
// failing call; as one_call of the thread-per-cell kernel.
template <int METHOD>
__device__ void run_cell(const unsigned* tab, const double* kc, double* sm, int lane,
                         const LaunchArgs& a, int cell) {
  constexpr int S = make_tableau(METHOD).S;
  using L = Cell<S>;
  const long ld = a.ld;
  CellEnv env;
  load_env(env, a.temp, a.cfactor, a.sun, a.fix, ld, cell);
  for (int i = lane; i < NVAR; i += 32) sm[L::V0 + i] = a.var[i * ld + cell];
  if (lane < NFIX_TRUE) {
    sm[L::V0 + NVAR + lane] = env.fix[lane];
    sm[L::V1 + NVAR + lane] = env.fix[lane];
  }
  if (lane == 0) {
    sm[L::V0 + K::ONE] = 1.0;
    sm[L::V1 + K::ONE] = 1.0;
  }
  double t0 = a.tstart[cell];
  __syncwarp();
  // rate constants (fixed for the call) by lane 0, staged in the matrix area
  double* rc = sm + L::JVS;
  if (lane == 0) {
    kpp_rconst_static(rc, t0, env.temp, env.cfactor, 0.0, sm + L::V0, env.fix);
    if (env.sun_fixed >= 0.0)
      kpp_rconst_sun(rc, t0, env.temp, env.cfactor, env.sun_fixed, sm + L::V0, env.fix);
  }
  __syncwarp();
  Weights w;
  weights<K::RF>(tab, K::O_WF, kc, rc, w.f, lane);
  weights<K::RJ>(tab, K::O_WJ, kc, rc, w.j, lane);
  __syncwarp();

  double rpar2 = a.hstart ? a.hstart[cell] : a.rpar[2];
  const int ncalls = a.nchain > 0 ? a.nchain : 1;
  for (int k = 0; k < ncalls; k++) {
    const double t1 = a.nchain > 0 ? t0 + a.chain_dt : a.tend[cell];
    Stats st = {0, 0, 0, 0, 0, 0, 0, 0};
    double texit = 0.0, hexit = 0.0;
    const int ierr = rosenbrock<METHOD>(tab, kc, w, sm, lane, t0, t1, a, rpar2, st, texit, hexit);
    if (lane == 0) {
      const int sv[8] = {st.nfun, st.njac, st.nstp, st.nacc, st.nrej, st.ndec, st.nsol, st.nsng};
      if (k == 0) {
        a.ierr[cell] = ierr;
        for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] = sv[i];
      } else {
        if (a.ierr[cell] == KPP_B200_IERR_SUCCESS) a.ierr[cell] = ierr;
        for (int i = 0; i < 8; i++) a.istatus[i * ld + cell] += sv[i];
      }
      a.rstatus[cell] = texit;
      a.rstatus[ld + cell] = hexit;
    }
    rpar2 = hexit;  // STEPMIN = RPAR[11]
    t0 = t1;        // TIME += DT
  }
  __syncwarp();
  for (int i = lane; i < NVAR; i += 32) a.var[i * ld + cell] = sm[L::V0 + i];
  __syncwarp();
}

// One CTA per SM: the tables are staged once, then each warp integrates cells
// one after another -- grid-stride over cells, or (QUEUE) the next cell of the
// work queue in the caller's order, so long and short cells balance.
template <int METHOD, bool QUEUE>
__global__ void __launch_bounds__(32 * warps_per_cta<make_tableau(METHOD).S>(), 1)
kernel(const LaunchArgs a) {
  constexpr int S = make_tableau(METHOD).S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned* tab = reinterpret_cast<unsigned*>(smem_raw);
  double* kc = reinterpret_cast<double*>(smem_raw + kTabBytes);
  double* cells = reinterpret_cast<double*>(smem_raw + kTablesBytes);
  for (int i = threadIdx.x; i < K::TAB_WORDS; i += blockDim.x) tab[i] = K::tab[i];
  for (int i = threadIdx.x; i < K::NKC; i += blockDim.x) kc[i] = K::kc[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* sm = cells + (size_t)warp * Cell<S>::TOTAL;
  if (QUEUE) {
    for (;;) {
      int pos = 0;
      if (lane == 0) pos = atomicAdd(a.queue, 1);
      pos = __shfl_sync(0xffffffffu, pos, 0);
      if (pos >= a.ncells) break;
      run_cell<METHOD>(tab, kc, sm, lane, a, a.order ? a.order[pos] : pos);
    }
  } else {
    const int wpb = blockDim.x >> 5;
    for (long c = (long)blockIdx.x * wpb + warp; c < a.ncells; c += (long)gridDim.x * wpb)
      run_cell<METHOD>(tab, kc, sm, lane, a, (int)c);
  }
}

}  // namespace coop
