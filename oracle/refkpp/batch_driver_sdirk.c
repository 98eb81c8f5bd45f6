/*~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
  Batch driver for the reference's own KPP-generated C model with the
  reference SDIRK integrator (#INTEGRATOR sdirk, int/sdirk.c).

  ORACLE INFRASTRUCTURE ONLY -- built by oracle/build_ref.sh into
  oracle/_ref/<mech>_sdirk/libkppsd_<mech>.so and loaded only by tests.

  Given to the generator with #DRIVER (src/gen.c:2564-2581) in place of the
  stock drv/general.c: it loops over a batch of independent cells, sets the
  generator's globals for each cell (C = VAR|FIX, TEMP, CFACTOR, TIME) and
  calls SDIRK(NVAR, Tstart, Tend, VAR, RTOL, ATOL, RCNTRL, ICNTRL, RSTATUS,
  ISTATUS) as INTEGRATE does (int/sdirk.c:92-166), with the caller's ICNTRL /
  RCNTRL and with ISTATUS / RSTATUS cleared before every call (INTEGRATE's
  arrays are fresh locals).  Per-cell sunlight as in batch_driver.c.

  Array layout: structure of arrays, cell index fastest, leading dimension ld.
  ISTATUS[1..8] and RSTATUS[1..3] (the integrator's Fortran-style slots) come
  back as rows 0..7 of istatus and 0..2 of rstatus.
~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~*/

double kppref_sun_override = -1.0;
int kppref_sun_ulps = 0;

/* Test knob: every evaluation moves SUN by one ulp up (1) or down (-1). */
void kppsd_set_sun_ulps(int u) { kppref_sun_ulps = u; }

/* The integrator's pow() in the libkppsd_<mech>_pw.so build (pow_knob.h
   force-included): libm's pow, moved one ulp up (1) or down (-1) on request.
   A constant exponent 2 gives x*x, as the compiler folds pow(x, 2) in the
   plain build, so that the knob at 0 reproduces the plain build bit for bit. */
static int kppref_pow_ulps = 0;
void kppref_set_pow_ulps(int u) { kppref_pow_ulps = u; }
/* Knob 1 / -1: every result one ulp up / down.  Knob 2 / 3: one ulp up,
   down or not, a direction hashed from the arguments (two different
   hashes), as a pow whose last-ulp error varies from call to call does:
   where the integrator's discrete decisions (accept, reuse the LU, Newton
   converged) sit on a pow result, such errors change the step sequence. */
double kppref_pow(double x, double y, int square)
{
  double r = square ? x * x : pow(x, y);
  if (kppref_pow_ulps == 1) r = nextafter(r, HUGE_VAL);
  if (kppref_pow_ulps == -1) r = nextafter(r, -HUGE_VAL);
  if (kppref_pow_ulps >= 2) {
    unsigned long long a, b, h;
    memcpy(&a, &x, 8);
    memcpy(&b, &y, 8);
    h = (a * 0x9E3779B97F4A7C15ull) ^ (b + (kppref_pow_ulps == 2 ? 0x632BE59BD9B4E019ull
                                                                  : 0xD1B54A32D192ED03ull));
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    if (h % 3 == 1) r = nextafter(r, HUGE_VAL);
    if (h % 3 == 2) r = nextafter(r, -HUGE_VAL);
  }
  return r;
}

/* Update_SUN's cos() in the same build (cos_knob.h force-included into the
   Rates file): libm's cos, moved one ulp up (1) or down (-1) on request.
   Near sunrise and sunset SUN = (1 + cos)/2 cancels, so one ulp of the
   cosine is a large relative change of SUN there. */
static int kppref_cos_ulps = 0;
void kppref_set_cos_ulps(int u) { kppref_cos_ulps = u; }
double kppref_cos(double x)
{
  double r = cos(x);
  if (kppref_cos_ulps > 0) r = nextafter(r, HUGE_VAL);
  if (kppref_cos_ulps < 0) r = nextafter(r, -HUGE_VAL);
  return r;
}

int SDIRK(int N, double Tinitial, double Tfinal, double Y[], double RelTol[],
          double AbsTol[], double RCNTRL[], int ICNTRL[], double RSTATUS[],
          int ISTATUS[]);

/* SDIRK_Integrator reads stage vectors that a step did not write when its
   Newton iteration failed (the local Z of int/sdirk.c:516, summed by the
   error estimate at :716-733), so its result depends on what the stack held
   before the call.  The stack region the call is about to use is cleared
   first, so every call sees zeros there, as the device integrator does. */
static __attribute__((noinline)) void scrub_stack(void)
{
  char buf[(2 * LU_NONZERO + 16 * NVAR) * sizeof(double) + 16384];
  explicit_bzero(buf, sizeof buf);
}

int kppsd_dims(int *d)
{
  d[0] = NVAR; d[1] = NFIX; d[2] = NSPEC; d[3] = NREACT; d[4] = LU_NONZERO;
  return 0;
}

int kppsd_integrate(int ncells, int ld, double *var, const double *fix,
                    const double *temp, const double *cfactor, const double *sun,
                    const double *tstart, const double *tend, const double *atol,
                    const double *rtol, const int *icntrl, const double *rcntrl,
                    int *istatus, double *rstatus, int *ierr)
{
  double at[NVAR], rt[NVAR], rc[20], rs[20];
  int ic[20], is[20];
  int cell, i;
  const int nt = icntrl[1] == 0 ? NVAR : 1;  /* vector or scalar tolerances */
  for (i = 0; i < NVAR; i++) { at[i] = atol[i < nt ? i : 0]; rt[i] = rtol[i < nt ? i : 0]; }
  for (cell = 0; cell < ncells; cell++) {
    for (i = 0; i < 20; i++) { ic[i] = icntrl[i]; rc[i] = rcntrl[i]; is[i] = 0; rs[i] = 0.0; }
    for (i = 0; i < NVAR; i++) VAR[i] = var[(long)i * ld + cell];
    /* NSPEC - NVAR real fixed species (KPP pads NFIX to 1 when there are none) */
    for (i = 0; i < NSPEC - NVAR; i++) FIX[i] = fix[(long)i * ld + cell];
    TEMP = temp[cell];
    if (cfactor) CFACTOR = cfactor[cell];
    kppref_sun_override = sun ? sun[cell] : -1.0;
    TIME = tstart[cell];

    scrub_stack();
    ierr[cell] = SDIRK(NVAR, tstart[cell], tend[cell], VAR, rt, at, rc, ic, rs, is);

    for (i = 0; i < NVAR; i++) var[(long)i * ld + cell] = VAR[i];
    for (i = 0; i < 8; i++) istatus[(long)i * ld + cell] = is[1 + i];
    for (i = 0; i < 3; i++) rstatus[(long)i * ld + cell] = rs[1 + i];
  }
  return 0;
}
