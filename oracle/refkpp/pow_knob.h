/* Force-included (-include) into the reference SDIRK integrator for the
   libkppsd_<mech>_pw.so build (ORACLE INFRASTRUCTURE ONLY): math.h first,
   then every later pow() of the file becomes the driver's kppsd_pow, which
   returns libm's pow moved one ulp on request. */
#include <math.h>
double kppsd_pow(double x, double y);
#define pow kppsd_pow
