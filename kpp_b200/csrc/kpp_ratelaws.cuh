// Device versions of the KPP utility templates used inside the rate
// constants: the rate-law functions of util/UserRateLaws.c:9-78 and the
// diurnal sun function of util/UpdateSun.c:1-20.
//
// The reference declares the rate-law arguments `float` (the mechanism's
// numbers are single precision by KPP convention) and computes in double; the
// generated code converts every argument to float before the call, so these
// take float and widen exactly where the reference does.  The order of the
// double operations is the reference's.
#pragma once

__device__ __forceinline__ double kpp_arr_abc(double TEMP, float A0, float B0, float C0) {
  return (double)A0 * exp(-(double)B0 / TEMP) * pow((TEMP / 300.0), (double)C0);
}

__device__ __forceinline__ double kpp_arr_ab(double TEMP, float A0, float B0) {
  return (double)A0 * exp(-(double)B0 / TEMP);
}

__device__ __forceinline__ double kpp_arr_ac(double TEMP, float A0, float C0) {
  return (double)A0 * pow((TEMP / 300.0), (double)C0);
}

__device__ __forceinline__ double kpp_ep2(double TEMP, double CFACTOR, float A0, float C0,
                                          float A2, float C2, float A3, float C3) {
  double K0 = (double)A0 * exp(-(double)C0 / TEMP);
  double K2 = (double)A2 * exp(-(double)C2 / TEMP);
  double K3 = (double)A3 * exp(-(double)C3 / TEMP);
  K3 = K3 * CFACTOR * 1.0e+6;
  return K0 + K3 / (1.0 + K3 / K2);
}

__device__ __forceinline__ double kpp_ep3(double TEMP, double CFACTOR, float A1, float C1,
                                          float A2, float C2) {
  double K1 = (double)A1 * exp(-(double)C1 / TEMP);
  double K2 = (double)A2 * exp(-(double)C2 / TEMP);
  return K1 + K2 * (1.0e+6 * CFACTOR);
}

__device__ __forceinline__ double kpp_fall(double TEMP, double CFACTOR, float A0, float B0,
                                           float C0, float A1, float B1, float C1, float CF) {
  double K0 = (double)A0 * exp(-(double)B0 / TEMP) * pow((TEMP / 300.0), (double)C0);
  double K1 = (double)A1 * exp(-(double)B1 / TEMP) * pow((TEMP / 300.0), (double)C1);
  K0 = K0 * CFACTOR * 1.0e+6;
  K1 = K0 / K1;
  return (K0 / (1.0 + K1)) * pow((double)CF, (1.0 / (1.0 + pow((log10(K1)), 2))));
}

// ---------------------------------------------------------------------------
// Correctly rounded cosine on [-4, 4] for Update_SUN.
//
// The host reference calls the C library's cos(), which returns the correctly
// rounded result for all but a small fraction of arguments; a device cos with
// a larger error bound would perturb SUN -- and through it the photolysis
// rates -- at many more evaluations.  This version computes cos(x) to about
// 2^-100 relative accuracy in double-double arithmetic and rounds once, so it
// returns the correctly rounded value except when the exact result lies
// within ~2^-100 of a rounding boundary.
//   * argument reduction (Cody and Waite): x = k*pi/2 + r, |r| <= pi/4, with
//     pi/2 split into three doubles so that r is exact to ~2^-150; valid for
//     |k| <= 3, i.e. |x| <= 4 (k*P1 is then exact); Update_SUN only passes
//     |x| <= pi;
//   * cos(r) and sin(r) by their Taylor series (16 terms each), evaluated by
//     Horner's rule in double-double arithmetic (Knuth's TwoSum and Dekker's
//     FastTwoSum and exact product, here through an FMA; the double-double
//     operations as formulated for the QD library by Hida, Li and Bailey);
//   * cos(x) = cos(r), -sin(r), -cos(r), sin(r) for k = 0, 1, 2, 3 (mod 4).
// Constants: pi/2 and (-1)^n/(2n)!, (-1)^n/(2n+1)! rounded to double-double.
// ---------------------------------------------------------------------------
struct kpp_dd {
  double hi, lo;
};

__host__ __device__ __forceinline__ double kpp_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}

__host__ __device__ __forceinline__ kpp_dd kpp_two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  return {s, e};
}

__host__ __device__ __forceinline__ kpp_dd kpp_fast_two_sum(double a, double b) {
  double s = a + b;
  return {s, b - (s - a)};
}

__host__ __device__ __forceinline__ kpp_dd kpp_dd_add(kpp_dd x, kpp_dd y) {
  kpp_dd s = kpp_two_sum(x.hi, y.hi);
  kpp_dd t = kpp_two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = kpp_fast_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return kpp_fast_two_sum(s.hi, s.lo);
}

__host__ __device__ __forceinline__ kpp_dd kpp_dd_mul(kpp_dd x, kpp_dd y) {
  double p = x.hi * y.hi;
  double e = kpp_fma(x.hi, y.hi, -p);
  e += x.hi * y.lo + x.lo * y.hi;
  return kpp_fast_two_sum(p, e);
}

__host__ __device__ inline double kpp_cos_cr(double x) {
  const double P1 = 1.5707963267948966, P2 = 6.123233995736766e-17,
               P3 = -1.4973849048591698e-33;
  const double kc[17][2] = {
      {1.0, 0.0}, {-0.5, 0.0}, {0.041666666666666664, 2.3129646346357427e-18},
      {-0.001388888888888889, 5.300543954373577e-20}, {2.48015873015873e-05, 2.1511947866775882e-23},
      {-2.755731922398589e-07, -2.3767714622250297e-23}, {2.08767569878681e-09, -1.20734505911326e-25},
      {-1.1470745597729725e-11, -2.0655512752830745e-28}, {4.779477332387385e-14, 4.399205485834081e-31},
      {-1.5619206968586225e-16, -1.1910679660273754e-32}, {4.110317623312165e-19, 1.4412973378659527e-36},
      {-8.896791392450574e-22, 7.911402614872376e-38}, {1.6117375710961184e-24, -3.6846573564509766e-41},
      {-2.4795962632247976e-27, 1.2953730964765229e-43}, {3.279889237069838e-30, 1.5117542744029879e-46},
      {-3.7699876288159054e-33, -2.5870347832750324e-49}, {3.8003907548547434e-36, 1.7457158024652518e-52}};
  const double ks[17][2] = {
      {1.0, 0.0}, {-0.16666666666666666, -9.25185853854297e-18},
      {0.008333333333333333, 1.1564823173178714e-19}, {-0.0001984126984126984, -1.7209558293420705e-22},
      {2.7557319223985893e-06, -1.858393274046472e-22}, {-2.505210838544172e-08, 1.448814070935912e-24},
      {1.6059043836821613e-10, 1.2585294588752098e-26}, {-7.647163731819816e-13, -7.03872877733453e-30},
      {2.8114572543455206e-15, 1.6508842730861433e-31}, {-8.22063524662433e-18, -2.2141894119604265e-34},
      {1.9572941063391263e-20, -1.3643503830087908e-36}, {-3.868170170630684e-23, 8.843177655482344e-40},
      {6.446950284384474e-26, -1.9330404233703465e-42}, {-9.183689863795546e-29, -1.4303150396787322e-45},
      {1.1309962886447716e-31, 1.0498015412959506e-47}, {-1.216125041553518e-34, -5.586290567888806e-51},
      {1.151633562077195e-37, -6.09957445788454e-54}};
  double kf = rint(x * 0.6366197723675814);
  int k = (int)kf;
  kpp_dd r = kpp_two_sum(x, -kf * P1);  // k*P1 is exact for |k| <= 3
  r = kpp_dd_add(r, {-kf * P2, 0.0});
  r = kpp_dd_add(r, {-kf * P3, 0.0});
  kpp_dd r2 = kpp_dd_mul(r, r);
  const bool use_sin = (k & 1) != 0;
  kpp_dd p = use_sin ? kpp_dd{ks[16][0], ks[16][1]} : kpp_dd{kc[16][0], kc[16][1]};
  for (int n = 15; n >= 0; n--) {
    kpp_dd c = use_sin ? kpp_dd{ks[n][0], ks[n][1]} : kpp_dd{kc[n][0], kc[n][1]};
    p = kpp_dd_add(kpp_dd_mul(p, r2), c);
  }
  if (use_sin) p = kpp_dd_mul(p, r);
  double v = p.hi + p.lo;
  int q = k & 3;
  return (q == 1 || q == 2) ? -v : v;
}

// The cosine of Update_SUN (the host harness of the tests substitutes the C
// library's to compare generated code bit for bit with the reference).
#ifndef KPP_SUN_COS
#define KPP_SUN_COS kpp_cos_cr
#endif

// SUN in [0,1] from the model time: a cosine-shaped day between 4.5 h and
// 19.5 h local time, 0 at night (util/UpdateSun.c:1-20).
__device__ __forceinline__ double kpp_update_sun(double TIME) {
  const double PI = 3.14159265358979;
  const double SunRise = 4.5, SunSet = 19.5;
  double Thour = TIME / 3600.0;
  double Tlocal = Thour - (double)(((int)Thour / 24) * 24);
  if ((Tlocal >= SunRise) && (Tlocal <= SunSet)) {
    double Ttmp = (2.0 * Tlocal - SunRise - SunSet) / (SunSet - SunRise);
    if (Ttmp > 0) Ttmp = Ttmp * Ttmp;
    else Ttmp = -Ttmp * Ttmp;
    return (1.0 + KPP_SUN_COS(PI * Ttmp)) / 2.0;
  }
  return 0.0;
}

// ---------------------------------------------------------------------------
// kpp_pow_cr(x, y): x^y correctly rounded to nearest (to within a final
// double-double error of about 2^-98 relative, so misrounded only for
// arguments whose exact result lies that close to a rounding midpoint).  It
// is the pow() of the integrators' step-size and Newton controllers
// (KPP_POW), whose results decide whether a step is accepted, a Jacobian
// reused or a Newton iteration stopped: with a correctly rounded pow those
// decisions follow the reference's wherever the C library's pow (which the
// reference calls) is correctly rounded.  Method, in double-double
// arithmetic (the operations above):
//   * x = 2^e m with m in [1/sqrt(2), sqrt(2)) (frexp);
//   * log m = 2 atanh(s), s = (m - 1)/(m + 1), |s| <= 0.1716, by the series
//     sum s^(2n+1)/(2n+1) (terms n <= 10 in double-double, n = 11..21 in
//     double, where they are below 2^-53 of the sum);
//   * log x = e ln2 + log m with ln2 split in three parts (Cody and Waite's
//     reduction: the first has 42 bits, so e * part exactly for |e| < 2^11);
//   * t = y log x; exp t = 2^k exp(r), k = nearest integer to t / ln2,
//     r = t - k ln2 by the same three-part split; exp(r) = (1 + u)^16 with
//     u = expm1(r / 16) by its Taylor series (terms n <= 7 in double-double,
//     the rest in double) and four squarings in the form u <- 2u + u^2;
//   * the double-double result rounded once to double, then scaled by 2^k.
// Special arguments (x or y zero, infinite or NaN; x negative with y not an
// integer) and results outside the normal range (|t| > 708) return the C
// library's pow(x, y): their values are exact (0, 1, inf, NaN) or, for the
// extremes, never reached by the controllers.  y = 1, 2, -1 and 1/2 are x,
// x*x, 1/x and sqrt(x), one correctly rounded operation each (which also
// settles their exact midpoint cases).  Constants: ln2 in three
// parts, 1/(2n+1) and 1/(n+1)! rounded to double-double.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ kpp_dd kpp_dd_mul_d(kpp_dd x, double y) {
  double p = x.hi * y;
  double e = kpp_fma(x.hi, y, -p);
  e += x.lo * y;
  return kpp_fast_two_sum(p, e);
}

__host__ __device__ __forceinline__ kpp_dd kpp_two_prod(double a, double b) {
  double p = a * b;
  return {p, kpp_fma(a, b, -p)};
}

__host__ __device__ inline double kpp_pow_cr(double x, double y) {
  if (y == 0.0 || x == 1.0) return 1.0;
  if (x != x || y != y) return x + y;
  const double ax = fabs(x);
  bool negate = false;
  if (x < 0.0) {
    if (y != trunc(y)) return pow(x, y);  // NaN
    negate = fabs(y) < 9007199254740992.0 && fmod(y, 2.0) != 0.0;
  }
  if (ax == 0.0 || isinf(ax) || isinf(y)) return pow(x, y);
  // exponents whose power is one IEEE operation, correctly rounded by itself
  if (y == 1.0) return x;
  if (y == 2.0) return x * x;
  if (y == -1.0) return 1.0 / x;
  if (y == 0.5) return sqrt(x);  // x > 0 here

  const double L1 = 0.6931471805598903, L2 = 5.497923018708371e-14, L3 = 1.94704509238075e-31;
  const double at[11][2] = {
      {1.0, 0.0}, {0.3333333333333333, 1.850371707708594e-17}, {0.2, -1.1102230246251566e-17},
      {0.14285714285714285, 7.93016446160826e-18}, {0.1111111111111111, 6.1679056923619804e-18},
      {0.09090909090909091, -2.523234146875356e-18}, {0.07692307692307693, -4.270088556250602e-18},
      {0.06666666666666667, 9.251858538542971e-19}, {0.058823529411764705, 8.163404592832033e-19},
      {0.05263157894736842, 2.921639538487254e-18}, {0.047619047619047616, 2.64338815386942e-18}};
  const double ex[8][2] = {
      {1.0, 0.0}, {0.5, 0.0}, {0.16666666666666666, 9.25185853854297e-18},
      {0.041666666666666664, 2.3129646346357427e-18}, {0.008333333333333333, 1.1564823173178714e-19},
      {0.001388888888888889, -5.300543954373577e-20}, {0.0001984126984126984, 1.7209558293420705e-22},
      {2.48015873015873e-05, 2.1511947866775882e-23}};

  // log x
  int e;
  double m = frexp(ax, &e);
  if (m < 0.7071067811865476) {
    m *= 2.0;
    e -= 1;
  }
  const double num = m - 1.0;  // exact: m in [0.5, 2]
  const kpp_dd den = kpp_two_sum(m, 1.0);
  kpp_dd s;
  {
    double q1 = num / den.hi;
    kpp_dd r = kpp_dd_add({num, 0.0}, kpp_dd_mul_d(den, -q1));
    double q2 = r.hi / den.hi;
    r = kpp_dd_add(r, kpp_dd_mul_d(den, -q2));
    double q3 = r.hi / den.hi;
    s = kpp_dd_add(kpp_fast_two_sum(q1, q2), {q3, 0.0});
  }
  const kpp_dd s2 = kpp_dd_mul(s, s);
  double tail = 1.0 / 43.0;
  for (int n = 20; n >= 11; n--) tail = tail * s2.hi + 1.0 / (double)(2 * n + 1);
  kpp_dd p = kpp_dd_add(kpp_dd_mul_d(s2, tail), {at[10][0], at[10][1]});
  for (int n = 9; n >= 0; n--) p = kpp_dd_add(kpp_dd_mul(p, s2), {at[n][0], at[n][1]});
  kpp_dd lm = kpp_dd_mul(s, p);
  lm.hi *= 2.0;
  lm.lo *= 2.0;
  const double de = (double)e;
  kpp_dd lx = kpp_dd_add(kpp_two_prod(de, L2), {de * L3, 0.0});
  lx = kpp_dd_add(kpp_dd_add({de * L1, 0.0}, lx), lm);

  // t = y log x, exp t
  const kpp_dd t = kpp_dd_mul_d(lx, y);
  if (!(fabs(t.hi) <= 708.0)) return pow(x, y);
  const double kf = rint(t.hi * 1.4426950408889634);
  kpp_dd r = kpp_two_sum(t.hi - kf * L1, t.lo);  // t.hi - kf*L1 is exact
  r = kpp_dd_add(r, kpp_two_prod(-kf, L2));
  r = kpp_dd_add(r, {-kf * L3, 0.0});
  r.hi *= 0.0625;
  r.lo *= 0.0625;
  double et = 1.1470745597729725e-11;
  const double tcoef[5] = {2.7557319223985893e-06, 2.755731922398589e-07, 2.505210838544172e-08,
                           2.08767569878681e-09, 1.6059043836821613e-10};
  for (int n = 4; n >= 0; n--) et = et * r.hi + tcoef[n];
  kpp_dd q = kpp_dd_add(kpp_dd_mul_d(r, et), {ex[7][0], ex[7][1]});
  for (int n = 6; n >= 0; n--) q = kpp_dd_add(kpp_dd_mul(q, r), {ex[n][0], ex[n][1]});
  kpp_dd u = kpp_dd_mul(r, q);
  for (int i = 0; i < 4; i++) u = kpp_dd_add({2.0 * u.hi, 2.0 * u.lo}, kpp_dd_mul(u, u));
  const kpp_dd E = kpp_dd_add({1.0, 0.0}, u);
  const double v = ldexp(E.hi, (int)kf);
  return negate ? -v : v;
}

// The pow of the integrators' controllers (the host harness of the tests
// substitutes the C library's to compare with the reference bit for bit).
#ifndef KPP_POW
#define KPP_POW kpp_pow_cr
#endif
