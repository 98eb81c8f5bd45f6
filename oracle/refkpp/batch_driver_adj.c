/*~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
  Batch driver for the reference's own KPP-generated C model with the
  reference Rosenbrock adjoint integrator (#INTEGRATOR rosenbrock_adj,
  int/rosenbrock_adj.c) and the generated Hessian (#HESSIAN ON).

  ORACLE INFRASTRUCTURE ONLY -- built by oracle/build_ref.sh into
  oracle/_ref/<mech>_adj/libkppadj_<mech>.so and loaded only by tests.

  Given to the generator with #DRIVER (src/gen.c:2564-2581) in place of the
  stock drv/general_adj.c: for each cell of a batch it sets the generator's
  globals (C = VAR|FIX, TEMP, CFACTOR, TIME) and calls RosenbrockADJ(VAR,
  NADJ, Lambda, Tstart, Tend, ATOL, RTOL, ATOL_adj, RTOL_adj, RCNTRL, ICNTRL,
  RSTATUS, ISTATUS) with the caller's controls, as INTEGRATE_ADJ does
  (int/rosenbrock_adj.c:124-189) but with controls of the caller's choice.
  The checkpoint capacity `bufsize` (the global of int/rosenbrock_adj.c:30,
  which also sets the default step limit bufsize - 1) is the caller's.
  Per-cell sunlight as in batch_driver.c.

  Array layout: structure of arrays, cell index fastest, leading dimension ld;
  lambda has NADJ * NVAR rows (adjoint m's entry i in row m * NVAR + i).
  ISTATUS[1..8] and RSTATUS[1..3] come back as rows 0..7 of istatus and 0..2
  of rstatus.
~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~*/
#include <stdlib.h>
#include <string.h>

double kppref_sun_override = -1.0;
int kppref_sun_ulps = 0;
extern int bufsize;

void kppadj_set_sun_ulps(int u) { kppref_sun_ulps = u; }

/* The integrator's pow() in the _pw build (pow_knob.h force-included):
   libm's pow, moved one ulp up (1) or down (-1) on request; a constant
   exponent 2 gives x*x, as the compiler folds pow(x, 2) in the plain build. */
static int kppref_pow_ulps = 0;
void kppref_set_pow_ulps(int u) { kppref_pow_ulps = u; }
double kppref_pow(double x, double y, int square)
{
  double r = square ? x * x : pow(x, y);
  if (kppref_pow_ulps > 0) r = nextafter(r, HUGE_VAL);
  if (kppref_pow_ulps < 0) r = nextafter(r, -HUGE_VAL);
  return r;
}

/* Update_SUN's cos() in the same build (cos_knob.h). */
static int kppref_cos_ulps = 0;
void kppref_set_cos_ulps(int u) { kppref_cos_ulps = u; }
double kppref_cos(double x)
{
  double r = cos(x);
  if (kppref_cos_ulps > 0) r = nextafter(r, HUGE_VAL);
  if (kppref_cos_ulps < 0) r = nextafter(r, -HUGE_VAL);
  return r;
}

int RosenbrockADJ(double Y[], int NADJ, double Lambda[][NVAR], double Tstart, double Tend,
                  double AbsTol[], double RelTol[], double AbsTol_adj[][NVAR],
                  double RelTol_adj[][NVAR], double RCNTRL[], int ICNTRL[], double RSTATUS[],
                  int ISTATUS[]);

int kppadj_dims(int *d)
{
  d[0] = NVAR; d[1] = NFIX; d[2] = NSPEC; d[3] = NREACT; d[4] = LU_NONZERO;
  return 0;
}

int kppadj_integrate(int ncells, int ld, double *var, const double *fix,
                     const double *temp, const double *cfactor, const double *sun,
                     const double *tstart, const double *tend, const double *atol,
                     const double *rtol, int nadj, double *lambda, const int *icntrl,
                     const double *rcntrl, int nbuf, int *istatus, double *rstatus, int *ierr)
{
  double at[NVAR], rt[NVAR], rc[20], rs[20];
  int ic[20], is[20];
  int cell, i, m;
  const int nt = icntrl[1] == 0 ? NVAR : 1;  /* vector or scalar tolerances */
  double (*lam)[NVAR] = calloc((size_t)(nadj > 0 ? nadj : 1), sizeof *lam);
  double (*atol_adj)[NVAR] = calloc((size_t)(nadj > 0 ? nadj : 1), sizeof *atol_adj);
  double (*rtol_adj)[NVAR] = calloc((size_t)(nadj > 0 ? nadj : 1), sizeof *rtol_adj);
  if (!lam || !atol_adj || !rtol_adj) return -1;
  bufsize = nbuf;
  for (i = 0; i < NVAR; i++) { at[i] = atol[i < nt ? i : 0]; rt[i] = rtol[i < nt ? i : 0]; }
  for (cell = 0; cell < ncells; cell++) {
    for (i = 0; i < 20; i++) { ic[i] = icntrl[i]; rc[i] = rcntrl[i]; is[i] = 0; rs[i] = 0.0; }
    for (i = 0; i < NVAR; i++) VAR[i] = var[(long)i * ld + cell];
    /* NSPEC - NVAR real fixed species (KPP pads NFIX to 1 when there are none) */
    for (i = 0; i < NSPEC - NVAR; i++) FIX[i] = fix[(long)i * ld + cell];
    for (m = 0; m < nadj; m++)
      for (i = 0; i < NVAR; i++) lam[m][i] = lambda[((long)m * NVAR + i) * ld + cell];
    TEMP = temp[cell];
    if (cfactor) CFACTOR = cfactor[cell];
    kppref_sun_override = sun ? sun[cell] : -1.0;
    TIME = tstart[cell];

    ierr[cell] = RosenbrockADJ(VAR, nadj, lam, tstart[cell], tend[cell], at, rt, atol_adj,
                               rtol_adj, rc, ic, rs, is);

    for (i = 0; i < NVAR; i++) var[(long)i * ld + cell] = VAR[i];
    for (m = 0; m < nadj; m++)
      for (i = 0; i < NVAR; i++) lambda[((long)m * NVAR + i) * ld + cell] = lam[m][i];
    for (i = 0; i < 8; i++) istatus[(long)i * ld + cell] = is[1 + i];
    for (i = 0; i < 3; i++) rstatus[(long)i * ld + cell] = rs[1 + i];
  }
  free(lam);
  free(atol_adj);
  free(rtol_adj);
  return 0;
}
