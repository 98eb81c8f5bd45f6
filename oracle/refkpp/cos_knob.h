/* Force-included (-include) into the generated Rates file (which holds
   Update_SUN) for the libkppsd_<mech>_pw.so and libkppref_<mech>_cs.so builds (ORACLE INFRASTRUCTURE
   ONLY): math.h first, then every later cos() of the file becomes the
   driver's kppref_cos, which returns libm's cos moved one ulp on request. */
#include <math.h>
double kppref_cos(double x);
#define cos kppref_cos
