/*~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~
  Batch driver for the reference's own KPP-generated C model.

  ORACLE INFRASTRUCTURE ONLY -- built by oracle/build_ref.sh into
  oracle/_ref/<mech>/libkppref_<mech>.so and loaded only by tests and the CPU
  baseline leg of bench.py.

  KPP's generator copies a driver given by path (`#DRIVER /path/name`,
  src/gen.c:2564-2581) into KPP_ROOT_Main.c through the same `sed` substitution
  it applies to every template (src/code.c:269-400).  This file replaces the
  stock box-model driver drv/general.c: instead of a time loop over one cell it
  loops over a batch of independent cells, sets the generator's globals for each
  cell (C = VAR|FIX, TEMP, CFACTOR, TIME) and calls the reference Rosenbrock
  integrator `Rosenbrock(VAR, Tstart, Tend, ATOL, RTOL, FunTemplate,
  JacTemplate, RPAR, IPAR)` exactly as INTEGRATE does (int/rosenbrock.c:94-133),
  but with the caller's IPAR/RPAR instead of INTEGRATE's hard-wired Rodas4.

  Per-cell sunlight: when `sun` is given, the mechanism's C_RCONST inline block
  (written by the build recipe) replaces the SUN that Update_SUN computed from
  TIME with that cell's value, so SUN is constant over the call.

  Array layout: structure of arrays, cell index fastest, leading dimension ld.
~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~~*/

double kppref_sun_override = -1.0;
int kppref_sun_ulps = 0;

/* Test knob: every evaluation moves SUN by one ulp up (1) or down (-1). */
void kppref_set_sun_ulps(int u) { kppref_sun_ulps = u; }

/* Update_SUN's cos() in the libkppref_<mech>_cs.so build (cos_knob.h
   force-included into the Rates file): libm's cos, moved one ulp up (1) or
   down (-1) on request.  Near sunrise and sunset SUN = (1 + cos)/2 cancels,
   so one ulp of the cosine is a large relative change of SUN there. */
static int kppref_cos_ulps = 0;
void kppref_set_cos_ulps(int u) { kppref_cos_ulps = u; }
double kppref_cos(double x)
{
  double r = cos(x);
  if (kppref_cos_ulps > 0) r = nextafter(r, HUGE_VAL);
  if (kppref_cos_ulps < 0) r = nextafter(r, -HUGE_VAL);
  return r;
}

int Rosenbrock(double Y[], double Tstart, double Tend, double AbsTol[],
               double RelTol[], void (*ode_Fun)(double, double[], double[]),
               void (*ode_Jac)(double, double[], double[]), double RPAR[],
               int IPAR[]);
void FunTemplate(double T, double Y[], double Ydot[]);
void JacTemplate(double T, double Y[], double Jcb[]);
void Initialize();
void Update_SUN();
void Update_RCONST();

/* Sizes of the generated model: NVAR, NFIX, NSPEC, NREACT, LU_NONZERO. */
int kppref_dims(int *d)
{
  d[0] = NVAR; d[1] = NFIX; d[2] = NSPEC; d[3] = NREACT; d[4] = LU_NONZERO;
  return 0;
}

const char *kppref_species_name(int i)
{
  return (i >= 0 && i < NSPEC) ? SPC_NAMES[i] : "";
}

/* Sparse LU pattern written by the generator (KPP_ROOT_JacobianSP.c). */
int kppref_lu_pattern(int *irow, int *icol, int *crow, int *diag)
{
  int i;
  for (i = 0; i < LU_NONZERO; i++) { irow[i] = LU_IROW[i]; icol[i] = LU_ICOL[i]; }
  for (i = 0; i <= NVAR; i++) { crow[i] = LU_CROW[i]; diag[i] = LU_DIAG[i]; }
  return 0;
}

/* Initial concentrations from #INITVALUES (KPP_ROOT_Initialize.c) and the
   generator's CFACTOR. */
int kppref_initial_values(double *c, double *cfactor)
{
  int i;
  Initialize();
  for (i = 0; i < NSPEC; i++) c[i] = C[i];
  *cfactor = CFACTOR;
  return 0;
}

static void set_cell_globals(int cell, int ld, const double *fix,
                             const double *temp, const double *cfactor,
                             const double *sun, double t)
{
  int i;
  /* NSPEC - NVAR real fixed species: with none, KPP still sets NFIX = 1 and
     FIX[0] would lie past the end of C[NSPEC] */
  for (i = 0; i < NSPEC - NVAR; i++) FIX[i] = fix[(long)i * ld + cell];
  TEMP = temp[cell];
  if (cfactor) CFACTOR = cfactor[cell];
  kppref_sun_override = sun ? sun[cell] : -1.0;
  TIME = t;
}

/* Reaction-rate constants and ODE right-hand side / Jacobian of one cell at
   time t, through the generated FunTemplate/JacTemplate path.  The cell's
   concentrations are the model's VAR, as when INTEGRATE calls Rosenbrock:
   rate constants that read the concentrations (Update_RCONST sees C) see
   them. */
int kppref_fun_jac(const double *var, const double *fix, double temp,
                   double cfactor, double sun, double t, double *rconst,
                   double *vdot, double *jvs)
{
  double *y = VAR;
  int i;
  for (i = 0; i < NVAR; i++) y[i] = var[i];
  set_cell_globals(0, 1, fix, &temp, &cfactor, sun >= 0.0 ? &sun : 0, t);
  if (vdot) FunTemplate(t, y, vdot);
  if (jvs) JacTemplate(t, y, jvs);
  if (rconst) {
    Update_SUN();
    Update_RCONST();
    for (i = 0; i < NREACT; i++) rconst[i] = RCONST[i];
  }
  return 0;
}

/* Integrate cells [0, ncells) from tstart[c] to tend[c].
     var     [NVAR][ld]  in/out concentrations
     fix     [NFIX][ld]  fixed species
     temp    [ld]        temperature
     cfactor [ld]|NULL   conversion factor (NULL keeps the generator's value)
     sun     [ld]|NULL   per-cell SUN (NULL: Update_SUN from TIME)
     tstart, tend [ld]
     atol, rtol          [NVAR] (ipar[1]==0) or scalar (ipar[1]!=0)
     ipar[20], rpar[20]  integrator controls, C indexing of int/rosenbrock.c
     hstart  [ld]|NULL   per-cell starting step (overrides rpar[2])
     istatus [8][ld]     IPAR[10..17] after the call
     rstatus [2][ld]     RPAR[10..11] (Texit, Hexit)
     ierr    [ld]        return value of Rosenbrock                        */
int kppref_integrate(int ncells, int ld, double *var, const double *fix,
                     const double *temp, const double *cfactor,
                     const double *sun, const double *tstart,
                     const double *tend, const double *atol,
                     const double *rtol, const int *ipar_in,
                     const double *rpar_in, const double *hstart,
                     int *istatus, double *rstatus, int *ierr)
{
  static double atol_g[NVAR], rtol_g[NVAR];
  double rpar[20];
  int ipar[20];
  int cell, i, ntol;

  ntol = (ipar_in[1] == 0) ? NVAR : 1;
  for (i = 0; i < ntol; i++) { atol_g[i] = atol[i]; rtol_g[i] = rtol[i]; }

  for (cell = 0; cell < ncells; cell++) {
    for (i = 0; i < 20; i++) { ipar[i] = ipar_in[i]; rpar[i] = rpar_in[i]; }
    for (i = 10; i < 20; i++) { ipar[i] = 0; rpar[i] = 0.0; }
    if (hstart) rpar[2] = hstart[cell];
    for (i = 0; i < NVAR; i++) VAR[i] = var[(long)i * ld + cell];
    set_cell_globals(cell, ld, fix, temp, cfactor, sun, tstart[cell]);

    ierr[cell] = Rosenbrock(VAR, tstart[cell], tend[cell], atol_g, rtol_g,
                            &FunTemplate, &JacTemplate, rpar, ipar);

    for (i = 0; i < NVAR; i++) var[(long)i * ld + cell] = VAR[i];
    for (i = 0; i < 8; i++) istatus[(long)i * ld + cell] = ipar[10 + i];
    rstatus[cell] = rpar[10];
    rstatus[(long)ld + cell] = rpar[11];
  }
  return 0;
}
