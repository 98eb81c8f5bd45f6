// Division by a divisor whose reciprocal is known.
//
// The backward substitution divides every row by its diagonal entry, four
// times per factorisation (once per Rosenbrock stage), on the critical path of
// the solve.  With y = RN(1/b) computed once per factorisation, each quotient
// takes three operations by Markstein's correction step (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Develop. 34(1), 1990): q0 = RN(a*y), r = a - b*q0 (exact, one
// FMA), q = RN(q0 + r*y).  For binary64 with round-to-nearest, q is the
// correctly rounded a/b -- the value the division instruction sequence gives --
// as long as no intermediate leaves the normal range.  The range guard keeps
// both operands within 2^-300 .. 2^300 (a zero, subnormal, infinite or NaN
// operand falls outside it) and uses a / b otherwise.  A device self-test of
// the library (kpp_b200_check_division) compares it with a / b on billions of
// operands, adversarial divisors included.
#pragma once

// Both operands inside the guarded range (biased exponents 723..1322).
__device__ __forceinline__ bool kpp_div_recip_ok(double a, double b) {
  const unsigned ea = ((unsigned)__double2hiint(a) >> 20) & 0x7FFu;
  const unsigned eb = ((unsigned)__double2hiint(b) >> 20) & 0x7FFu;
  return ea - 723u < 600u && eb - 723u < 600u;
}

// Markstein's correction step; equal to a / b when kpp_div_recip_ok(a, b).
__device__ __forceinline__ double kpp_div_recip_fast(double a, double b, double y) {
  const double q0 = a * y;
  const double r = __fma_rn(-b, q0, a);
  return __fma_rn(r, y, q0);
}

__device__ __forceinline__ double kpp_div_recip(double a, double b, double y) {
  return kpp_div_recip_ok(a, b) ? kpp_div_recip_fast(a, b, y) : a / b;
}
