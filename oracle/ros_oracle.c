/* CPU restatement of the reference Rosenbrock INTEGRATE path.
 *
 * ORACLE INFRASTRUCTURE ONLY -- test and CPU-baseline code.  Nothing in the
 * product (kpp_b200/, include/) links, loads or calls this file; the product
 * path fails loudly when its CUDA library is missing instead of falling back
 * to any CPU code.
 *
 * What it is: a line-by-line restatement of the reference C
 * integrator int/rosenbrock.c together with the no-pivot sparse LU of
 * util/sutil.c:2-23, the BLAS-like helpers of util/blas.c it uses, and the
 * loop form of the generated KppSolve (src/gen.c:1960-2034).  It is compiled
 * by oracle/build_ref.sh into the same shared library as the reference's own
 * KPP-generated mechanism code, and gets the mechanism through the generated
 * FunTemplate / JacTemplate (Update_SUN + Update_RCONST + Fun / Jac_SP,
 * int/rosenbrock.c:1257-1296) and the generated LU_* sparsity arrays.
 *
 * How it is pinned: tests/test_oracle_pin.py runs this restatement and the
 * reference's own Rosenbrock (oracle/refkpp/batch_driver.c) on the same cells
 * and requires bit-identical results, statistics and error codes.
 *
 * Operation order is kept exactly (WAXPY's skip when alpha == 0, the MIN/MAX
 * macro forms and their NaN behaviour, SQRT = pow(x, 0.5), the left-to-right
 * sums), so that a same-compiler build reproduces the reference bit for bit.
 *
 * The build compiles this file with the generated model headers force-included
 * (NVAR, LU_NONZERO, LU_CROW/LU_DIAG/LU_ICOL, FunTemplate, ...).
 */
#include <math.h>
#include <stdio.h>
#include <string.h>

/* int/rosenbrock.c:1-11 */
#define OR_MAX(a, b) (((a) >= (b)) ? (a) : (b))
#define OR_MIN(b, c) (((b) < (c)) ? (b) : (c))
#define OR_ABS(x) (((x) >= 0) ? (x) : (-x))
#define OR_SQRT(d) (pow((d), 0.5))
#define OR_ZERO 0.0
#define OR_ONE 1.0
#define OR_HALF 0.5
#define OR_DELTAMIN 1.0e-6

void FunTemplate(double T, double Y[], double Ydot[]);
void JacTemplate(double T, double Y[], double Jcb[]);
extern double kppref_sun_override;

/* Test knob (0 = off, the default, bit-identical to the reference): move the
 * result of pow(Err, 1/ELO) in the step-size controller by one ulp up (1) or
 * down (-1), to measure how far a last-ulp difference of pow() moves the
 * results. */
static int kppor_pow_ulps = 0;
void kppor_set_pow_ulps(int u) { kppor_pow_ulps = u; }

static double or_pow_step(double err, double e) {
  double v = pow(err, e);
  if (kppor_pow_ulps > 0) v = nextafter(v, HUGE_VAL);
  if (kppor_pow_ulps < 0) v = nextafter(v, -HUGE_VAL);
  return v;
}

typedef struct {
  int nfun, njac, nstp, nacc, nrej, ndec, nsol, nsng;
} or_stats;

typedef struct {
  int S;
  double A[15], C[15], M[6], E[6], Alpha[6], Gamma[6], ELO;
  char NewF[6];
} or_method;

/* Tableaux: int/rosenbrock.c:779-1222 (Ros2, Ros3, Ros4, Rodas3, Rodas3_1,
 * Rodas4).  The published coefficients are the methods' definition and are
 * reproduced value for value. */
static void or_tableau(int method, or_method *m) {
  memset(m, 0, sizeof *m);
  switch (method) {
    case 1: { /* Ros2, :779-830 */
      double g = 1.70710678118655;
      m->S = 2;
      m->A[0] = 1.0 / g;
      m->C[0] = (-2.0) / g;
      m->NewF[0] = 1; m->NewF[1] = 1;
      m->M[0] = (3.0) / (2.0 * g); m->M[1] = (1.0) / (2.0 * g);
      m->E[0] = 1.0 / (2.0 * g); m->E[1] = 1.0 / (2.0 * g);
      m->ELO = 2.0;
      m->Alpha[0] = 0.0; m->Alpha[1] = 1.0;
      m->Gamma[0] = g; m->Gamma[1] = -g;
      break;
    }
    case 2: /* Ros3, :834-894 */
      m->S = 3;
      m->A[0] = 1.0; m->A[1] = 1.0; m->A[2] = 0.0;
      m->C[0] = -1.0156171083877702091975600115545;
      m->C[1] = 4.0759956452537699824805835358067;
      m->C[2] = 9.2076794298330791242156818474003;
      m->NewF[0] = 1; m->NewF[1] = 1; m->NewF[2] = 0;
      m->M[0] = 1.0;
      m->M[1] = 6.1697947043828245592553615689730;
      m->M[2] = -0.4277225654321857332623837380651;
      m->E[0] = 0.5;
      m->E[1] = -2.9079558716805469821718236208017;
      m->E[2] = 0.2235406989781156962736090927619;
      m->ELO = 3.0;
      m->Alpha[0] = 0.0;
      m->Alpha[1] = 0.43586652150845899941601945119356;
      m->Alpha[2] = 0.43586652150845899941601945119356;
      m->Gamma[0] = 0.43586652150845899941601945119356;
      m->Gamma[1] = 0.24291996454816804366592249683314;
      m->Gamma[2] = 2.1851380027664058511513169485832;
      break;
    case 3: /* Ros4, :898-972 */
      m->S = 4;
      m->A[0] = 0.2000000000000000e+01;
      m->A[1] = 0.1867943637803922e+01;
      m->A[2] = 0.2344449711399156;
      m->A[3] = m->A[1]; m->A[4] = m->A[2]; m->A[5] = 0.0;
      m->C[0] = -0.7137615036412310e+01;
      m->C[1] = 0.2580708087951457e+01;
      m->C[2] = 0.6515950076447975;
      m->C[3] = -0.2137148994382534e+01;
      m->C[4] = -0.3214669691237626;
      m->C[5] = -0.6949742501781779;
      m->NewF[0] = 1; m->NewF[1] = 1; m->NewF[2] = 1; m->NewF[3] = 0;
      m->M[0] = 0.2255570073418735e+01;
      m->M[1] = 0.2870493262186792;
      m->M[2] = 0.4353179431840180;
      m->M[3] = 0.1093502252409163e+01;
      m->E[0] = -0.2815431932141155;
      m->E[1] = -0.7276199124938920e-01;
      m->E[2] = -0.1082196201495311;
      m->E[3] = -0.1093502252409163e+01;
      m->ELO = 4.0;
      m->Alpha[0] = 0.0;
      m->Alpha[1] = 0.1145640000000000e+01;
      m->Alpha[2] = 0.6552168638155900;
      m->Alpha[3] = m->Alpha[2];
      m->Gamma[0] = 0.5728200000000000;
      m->Gamma[1] = -0.1769193891319233e+01;
      m->Gamma[2] = 0.7592633437920482;
      m->Gamma[3] = -0.1049021087100450;
      break;
    case 4: /* Rodas3, :976-1044 */
      m->S = 4;
      m->A[0] = 0.0; m->A[1] = 2.0; m->A[2] = 0.0;
      m->A[3] = 2.0; m->A[4] = 0.0; m->A[5] = 1.0;
      m->C[0] = 4.0; m->C[1] = 1.0; m->C[2] = -1.0;
      m->C[3] = 1.0; m->C[4] = -1.0; m->C[5] = -2.66666666666667;
      m->NewF[0] = 1; m->NewF[1] = 0; m->NewF[2] = 1; m->NewF[3] = 1;
      m->M[0] = 2.0; m->M[1] = 0.0; m->M[2] = 1.0; m->M[3] = 1.0;
      m->E[0] = 0.0; m->E[1] = 0.0; m->E[2] = 0.0; m->E[3] = 1.0;
      m->ELO = 3.0;
      m->Alpha[0] = 0.0; m->Alpha[1] = 0.0; m->Alpha[2] = 1.0; m->Alpha[3] = 1.0;
      m->Gamma[0] = 0.5; m->Gamma[1] = 1.5; m->Gamma[2] = 0.0; m->Gamma[3] = 0.0;
      break;
    case 7: /* Rodas3_1, :1048-1117 */
      m->S = 4;
      m->A[0] = 0.000000000000000; m->A[1] = 0.646601929740551;
      m->A[2] = 0.409567801987914; m->A[3] = 0.646601929740551;
      m->A[4] = 0.409567801987914; m->A[5] = 1.000000000000000;
      m->C[0] = 4.198495621784201; m->C[1] = 3.711590161613010;
      m->C[2] = -1.787771994729384; m->C[3] = 4.458898153216104;
      m->C[4] = -2.024095448516552; m->C[5] = -2.626700600119396;
      m->NewF[0] = 1; m->NewF[1] = 0; m->NewF[2] = 1; m->NewF[3] = 1;
      m->M[0] = 0.646601929740551; m->M[1] = 0.409567801987914;
      m->M[2] = 1.000000000000000; m->M[3] = 1.000000000000000;
      m->E[0] = 0.0; m->E[1] = 0.0; m->E[2] = 0.0; m->E[3] = 1.0;
      m->ELO = 3.0;
      m->Alpha[0] = 0.0; m->Alpha[1] = 0.0; m->Alpha[2] = 1.0; m->Alpha[3] = 1.0;
      m->Gamma[0] = 0.515000000000000; m->Gamma[1] = 1.628546001287715;
      m->Gamma[2] = 0.0; m->Gamma[3] = 0.0;
      break;
    case 5: /* Rodas4, :1121-1222 */
      m->S = 6;
      m->Alpha[0] = 0.000; m->Alpha[1] = 0.386; m->Alpha[2] = 0.210;
      m->Alpha[3] = 0.630; m->Alpha[4] = 1.000; m->Alpha[5] = 1.000;
      m->Gamma[0] = 0.2500000000000000; m->Gamma[1] = -0.1043000000000000;
      m->Gamma[2] = 0.1035000000000000; m->Gamma[3] = -0.3620000000000023e-01;
      m->Gamma[4] = 0.0; m->Gamma[5] = 0.0;
      m->A[0] = 0.1544000000000000e+01; m->A[1] = 0.9466785280815826;
      m->A[2] = 0.2557011698983284; m->A[3] = 0.3314825187068521e+01;
      m->A[4] = 0.2896124015972201e+01; m->A[5] = 0.9986419139977817;
      m->A[6] = 0.1221224509226641e+01; m->A[7] = 0.6019134481288629e+01;
      m->A[8] = 0.1253708332932087e+02; m->A[9] = -0.6878860361058950;
      m->A[10] = m->A[6]; m->A[11] = m->A[7]; m->A[12] = m->A[8];
      m->A[13] = m->A[9]; m->A[14] = 1.0;
      m->C[0] = -0.5668800000000000e+01; m->C[1] = -0.2430093356833875e+01;
      m->C[2] = -0.2063599157091915; m->C[3] = -0.1073529058151375;
      m->C[4] = -0.9594562251023355e+01; m->C[5] = -0.2047028614809616e+02;
      m->C[6] = 0.7496443313967647e+01; m->C[7] = -0.1024680431464352e+02;
      m->C[8] = -0.3399990352819905e+02; m->C[9] = 0.1170890893206160e+02;
      m->C[10] = 0.8083246795921522e+01; m->C[11] = -0.7981132988064893e+01;
      m->C[12] = -0.3152159432874371e+02; m->C[13] = 0.1631930543123136e+02;
      m->C[14] = -0.6058818238834054e+01;
      m->M[0] = m->A[6]; m->M[1] = m->A[7]; m->M[2] = m->A[8];
      m->M[3] = m->A[9]; m->M[4] = 1.0; m->M[5] = 1.0;
      m->E[5] = 1.0;
      m->NewF[0] = m->NewF[1] = m->NewF[2] = m->NewF[3] = m->NewF[4] = m->NewF[5] = 1;
      m->ELO = 4.0;
      break;
  }
}

/* WAXPY, util/blas.c:51-82: y <- y + alpha*x, skipped when alpha == 0. */
static void or_axpy(int n, double alpha, const double *x, double *y) {
  int i;
  if (alpha == OR_ZERO) return;
  for (i = 0; i < n; i++) y[i] = y[i] + alpha * x[i];
}

/* WLAMCH('E'), util/blas.c:150-183: unit roundoff by halving until 1+eps==1. */
static double or_wlamch(void) {
  double eps = pow(OR_HALF, 16), suma;
  volatile double one = OR_ONE;
  int i;
  for (i = 17; i <= 80; i++) {
    eps = eps * OR_HALF;
    suma = one + eps;
    if (suma <= OR_ONE) break;
  }
  return eps * 2.0;
}

/* KppDecomp, util/sutil.c:2-23: in-place no-pivot sparse LU in row order. */
static int or_decomp(double *jvs) {
  double w[NVAR];
  double a;
  int k, kk, j, jj;
  for (k = 0; k < NVAR; k++) {
    if (jvs[LU_DIAG[k]] == 0.0) return k + 1;
    for (kk = LU_CROW[k]; kk < LU_CROW[k + 1]; kk++) w[LU_ICOL[kk]] = jvs[kk];
    for (kk = LU_CROW[k]; kk < LU_DIAG[k]; kk++) {
      j = LU_ICOL[kk];
      a = -w[j] / jvs[LU_DIAG[j]];
      w[j] = -a;
      for (jj = LU_DIAG[j] + 1; jj < LU_CROW[j + 1]; jj++) w[LU_ICOL[jj]] += a * jvs[jj];
    }
    for (kk = LU_CROW[k]; kk < LU_CROW[k + 1]; kk++) jvs[kk] = w[LU_ICOL[kk]];
  }
  return 0;
}

/* KppSolve, generated by src/gen.c:1960-2034: forward substitution with the
 * unit lower factor, then backward substitution with the upper factor.  The
 * generated code writes each row as one left-to-right expression
 * x[i] = (x[i] - J*x[c] - ...) / J[diag]; the loop keeps that order. */
static void or_solve(const double *jvs, double *x) {
  int i, j;
  for (i = 0; i < NVAR; i++) {
    double s = x[i];
    if (LU_CROW[i] < LU_DIAG[i]) {
      for (j = LU_CROW[i]; j < LU_DIAG[i]; j++) s = s - jvs[j] * x[LU_ICOL[j]];
      x[i] = s;
    }
  }
  for (i = NVAR - 1; i >= 0; i--) {
    double s = x[i];
    for (j = LU_DIAG[i] + 1; j < LU_CROW[i + 1]; j++) s = s - jvs[j] * x[LU_ICOL[j]];
    x[i] = s / jvs[LU_DIAG[i]];
  }
}

/* ros_ErrorNorm, int/rosenbrock.c:632-659 */
static double or_error_norm(const double *y, const double *ynew, const double *yerr,
                            const double *atol, const double *rtol, int vectortol) {
  double err = OR_ZERO, scale, ymax;
  int i;
  for (i = 0; i < NVAR; i++) {
    ymax = OR_MAX(OR_ABS(y[i]), OR_ABS(ynew[i]));
    if (vectortol)
      scale = atol[i] + rtol[i] * ymax;
    else
      scale = atol[0] + rtol[0] * ymax;
    err = err + (yerr[i] * yerr[i]) / (scale * scale);
  }
  return OR_SQRT(err / (double)NVAR);
}

/* ros_FunTimeDerivative, int/rosenbrock.c:663-682 */
static void or_fun_time_derivative(double t, double roundoff, double *y,
                                   const double *fcn0, double *dfdt, or_stats *st) {
  double delta = OR_SQRT(roundoff) * OR_MAX(OR_DELTAMIN, OR_ABS(t));
  double inv;
  int i;
  FunTemplate(t + delta, y, dfdt);
  st->nfun++;
  or_axpy(NVAR, (-OR_ONE), fcn0, dfdt);
  inv = OR_ONE / delta;
  if (inv != OR_ONE)
    for (i = 0; i < NVAR; i++) dfdt[i] = inv * dfdt[i];
}

/* ros_PrepareMatrix, int/rosenbrock.c:686-737; returns 1 when singular */
static int or_prepare_matrix(double *h, int direction, double gam, const double *jac0,
                             double *ghimj, or_stats *st) {
  int i, ising, nconsecutive = 0;
  double ghinv;
  for (;;) {
    for (i = 0; i < LU_NONZERO; i++) ghimj[i] = -jac0[i];
    ghinv = OR_ONE / (direction * (*h) * gam);
    for (i = 0; i < NVAR; i++) ghimj[LU_DIAG[i]] = ghimj[LU_DIAG[i]] + ghinv;
    ising = or_decomp(ghimj);
    st->ndec++;
    if (ising == 0) return 0;
    st->nsng++;
    nconsecutive++;
    printf("\nWarning: LU Decomposition returned ising = %d\n", ising);
    if (nconsecutive <= 5)
      *h = (*h) * OR_HALF;
    else
      return 1;
  }
}

/* RosenbrockIntegrator, int/rosenbrock.c:450-627 */
static int or_integrator(double *y, double tstart, double tend, const double *atol,
                         const double *rtol, const or_method *m, int autonomous,
                         int vectortol, int max_no_steps, double roundoff, double hmin,
                         double hmax, double hstart, double facmin, double facmax,
                         double facrej, double facsafe, double *texit, double *hexit,
                         or_stats *st) {
  double ynew[NVAR], fcn0[NVAR], fcn[NVAR], dfdt[NVAR], jac0[LU_NONZERO],
      ghimj[LU_NONZERO], k[NVAR * 6], yerr[NVAR];
  double h, t, hnew, hc, hg, fac, tau, err;
  int direction, ioffset, j, istage, i;
  int reject_last = 0, reject_more = 0;

  t = tstart;
  *hexit = 0.0;
  h = OR_MIN(hstart, hmax);
  if (OR_ABS(h) <= 10.0 * roundoff) h = OR_DELTAMIN;
  direction = (tend >= tstart) ? +1 : -1;

  while (((direction > 0) && ((t - tend) + roundoff <= OR_ZERO)) ||
         ((direction < 0) && ((tend - t) + roundoff <= OR_ZERO))) {
    if (st->nstp > max_no_steps) {
      *texit = t;
      return -6;
    }
    if (((t + 0.1 * h) == t) || (h <= roundoff)) {
      *texit = t;
      return -7;
    }
    *hexit = h;
    h = OR_MIN(h, OR_ABS(tend - t));

    FunTemplate(t, y, fcn0);
    st->nfun++;
    if (!autonomous) or_fun_time_derivative(t, roundoff, y, fcn0, dfdt, st);
    JacTemplate(t, y, jac0);
    st->njac++;

    for (;;) { /* until the step is accepted */
      if (or_prepare_matrix(&h, direction, m->Gamma[0], jac0, ghimj, st)) {
        *texit = t;
        return -8;
      }
      for (istage = 1; istage <= m->S; istage++) {
        ioffset = NVAR * (istage - 1);
        if (istage == 1) {
          memcpy(fcn, fcn0, sizeof fcn);
        } else if (m->NewF[istage - 1]) {
          memcpy(ynew, y, sizeof ynew);
          for (j = 1; j <= istage - 1; j++)
            or_axpy(NVAR, m->A[(istage - 1) * (istage - 2) / 2 + j - 1], &k[NVAR * (j - 1)], ynew);
          tau = t + m->Alpha[istage - 1] * direction * h;
          FunTemplate(tau, ynew, fcn);
          st->nfun++;
        }
        memcpy(&k[ioffset], fcn, sizeof fcn);
        for (j = 1; j <= istage - 1; j++) {
          hc = m->C[(istage - 1) * (istage - 2) / 2 + j - 1] / (direction * h);
          or_axpy(NVAR, hc, &k[NVAR * (j - 1)], &k[ioffset]);
        }
        if ((!autonomous) && (m->Gamma[istage - 1])) {
          hg = direction * h * m->Gamma[istage - 1];
          or_axpy(NVAR, hg, dfdt, &k[ioffset]);
        }
        or_solve(ghimj, &k[ioffset]);
        st->nsol++;
      }

      memcpy(ynew, y, sizeof ynew);
      for (j = 1; j <= m->S; j++) or_axpy(NVAR, m->M[j - 1], &k[NVAR * (j - 1)], ynew);
      for (i = 0; i < NVAR; i++) yerr[i] = OR_ZERO;
      for (j = 1; j <= m->S; j++) or_axpy(NVAR, m->E[j - 1], &k[NVAR * (j - 1)], yerr);
      err = or_error_norm(y, ynew, yerr, atol, rtol, vectortol);

      fac = OR_MIN(facmax, OR_MAX(facmin, facsafe / or_pow_step(err, OR_ONE / m->ELO)));
      hnew = h * fac;

      st->nstp++;
      if ((err <= OR_ONE) || (h <= hmin)) {
        st->nacc++;
        memcpy(y, ynew, sizeof ynew);
        t += direction * h;
        hnew = OR_MAX(hmin, OR_MIN(hnew, hmax));
        if (reject_last) hnew = OR_MIN(hnew, h);
        reject_last = 0;
        reject_more = 0;
        h = hnew;
        break;
      } else {
        if (st->nacc >= 1) st->nrej++;
        if (reject_more) hnew = h * facrej;
        reject_more = reject_last;
        reject_last = 1;
        h = hnew;
      }
    }
  }
  *texit = t;
  return 1;
}

/* Rosenbrock, int/rosenbrock.c:137-446: control validation and defaults.
 * ipar/rpar use the C indexing of that file; ipar[10..17] and rpar[10..11]
 * receive the statistics, Texit and Hexit. */
static int or_rosenbrock(double *y, double tstart, double tend, const double *abstol,
                         const double *reltol, double *rpar, int *ipar) {
  or_method m;
  or_stats st;
  int max_no_steps, method, i, uplimtol, ierr, autonomous, vectortol;
  double roundoff, facmin, facmax, facrej, facsafe, hmin, hmax, hstart, hexit = 0, texit = 0;

  st.nfun = ipar[10]; st.njac = ipar[11]; st.nstp = ipar[12]; st.nacc = ipar[13];
  st.nrej = ipar[14]; st.ndec = ipar[15]; st.nsol = ipar[16]; st.nsng = ipar[17];

  autonomous = !(ipar[0] == 0);
  if (ipar[1] == 0) {
    vectortol = 1; uplimtol = NVAR;
  } else {
    vectortol = 0; uplimtol = 1;
  }
  max_no_steps = (ipar[2] == 0) ? 100000 : ipar[2];
  if (max_no_steps < 0) return -1;
  method = (ipar[3] == 0) ? 3 : ipar[3];
  if ((ipar[3] < 1) || (ipar[3] > 5)) return -2;
  roundoff = or_wlamch();
  hmin = rpar[0];
  if (rpar[0] < OR_ZERO) return -3;
  if (rpar[1] == OR_ZERO)
    hmax = OR_ABS(tend - tstart);
  else
    hmax = OR_MIN(OR_ABS(rpar[1]), OR_ABS(tend - tstart));
  if (rpar[1] < OR_ZERO) return -3;
  if (rpar[2] == OR_ZERO)
    hstart = OR_MAX(hmin, OR_DELTAMIN);
  else
    hstart = OR_MIN(OR_ABS(rpar[2]), OR_ABS(tend - tstart));
  if (rpar[2] < OR_ZERO) return -3;
  facmin = (rpar[3] == OR_ZERO) ? 0.2 : rpar[3];
  if (rpar[3] < OR_ZERO) return -4;
  facmax = (rpar[4] == OR_ZERO) ? 6.0 : rpar[4];
  if (rpar[4] < OR_ZERO) return -4;
  facrej = (rpar[5] == OR_ZERO) ? 0.1 : rpar[5];
  if (rpar[5] < OR_ZERO) return -4;
  facsafe = (rpar[6] == OR_ZERO) ? 0.9 : rpar[6];
  if (rpar[6] < OR_ZERO) return -4;
  for (i = 0; i < uplimtol; i++)
    if ((abstol[i] <= OR_ZERO) || (reltol[i] <= 10.0 * roundoff) || (reltol[i] >= OR_ONE))
      return -5;

  or_tableau(method, &m);
  ierr = or_integrator(y, tstart, tend, abstol, reltol, &m, autonomous, vectortol,
                       max_no_steps, roundoff, hmin, hmax, hstart, facmin, facmax, facrej,
                       facsafe, &texit, &hexit, &st);

  ipar[10] = st.nfun; ipar[11] = st.njac; ipar[12] = st.nstp; ipar[13] = st.nacc;
  ipar[14] = st.nrej; ipar[15] = st.ndec; ipar[16] = st.nsol; ipar[17] = st.nsng;
  rpar[10] = texit;
  rpar[11] = hexit;
  return ierr;
}

/* Batch entry with the argument list of kppref_integrate
 * (oracle/refkpp/batch_driver.c). */
int kppor_integrate(int ncells, int ld, double *var, const double *fix, const double *temp,
                    const double *cfactor, const double *sun, const double *tstart,
                    const double *tend, const double *atol, const double *rtol,
                    const int *ipar_in, const double *rpar_in, const double *hstart,
                    int *istatus, double *rstatus, int *ierr) {
  /* The cell is integrated in the model's VAR array, as INTEGRATE passes VAR
     to Rosenbrock (int/rosenbrock.c:116): rate constants that read the
     concentrations (Update_RCONST sees the global C) then see the accepted
     state, exactly as in the reference. */
  double *y = VAR;
  double rpar[20];
  int ipar[20];
  int cell, i;
  for (cell = 0; cell < ncells; cell++) {
    for (i = 0; i < 20; i++) { ipar[i] = ipar_in[i]; rpar[i] = rpar_in[i]; }
    for (i = 10; i < 20; i++) { ipar[i] = 0; rpar[i] = 0.0; }
    if (hstart) rpar[2] = hstart[cell];
    for (i = 0; i < NVAR; i++) y[i] = var[(long)i * ld + cell];
    /* NSPEC - NVAR real fixed species: with none, KPP still sets NFIX = 1
       and FIX[0] would lie past the end of C[NSPEC] */
    for (i = 0; i < NSPEC - NVAR; i++) FIX[i] = fix[(long)i * ld + cell];
    TEMP = temp[cell];
    if (cfactor) CFACTOR = cfactor[cell];
    kppref_sun_override = sun ? sun[cell] : -1.0;
    TIME = tstart[cell];

    ierr[cell] = or_rosenbrock(y, tstart[cell], tend[cell], atol, rtol, rpar, ipar);

    for (i = 0; i < NVAR; i++) var[(long)i * ld + cell] = y[i];
    for (i = 0; i < 8; i++) istatus[(long)i * ld + cell] = ipar[10 + i];
    rstatus[cell] = rpar[10];
    rstatus[(long)ld + cell] = rpar[11];
  }
  return 0;
}
