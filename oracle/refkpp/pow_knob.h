/* Force-included (-include) into the reference SDIRK or Runge-Kutta
   integrator for the libkppsd_<mech>_pw.so / libkpprk_<mech>_pw.so builds
   (ORACLE INFRASTRUCTURE ONLY): math.h first, then every later pow() of the
   file becomes the driver's kppref_pow, which returns libm's pow moved one
   ulp on request.  The third argument tells it the exponent is the constant
   2, which the compiler folds into x*x in the plain build. */
#include <math.h>
double kppref_pow(double x, double y, int square);
#define pow(x, y) kppref_pow((x), (y), __builtin_constant_p(y) && (y) == 2.0)
