/*
 * kpp_b200.h -- C ABI of the B200 batched Rosenbrock engine for KPP
 * mechanisms.
 *
 * One shared library per mechanism (libkpp_b200_<mechanism>.so), built from
 * the mechanism's KPP files by the kppcu mechanism compiler and the
 * hand-written sm_100a Rosenbrock kernel.  Every entry point takes plain
 * pointers and sizes; no CUDA or torch types appear in the signatures (the
 * stream is passed as `void *` holding a cudaStream_t, NULL = legacy default
 * stream).
 *
 * Layout of batched arrays: structure of arrays with the cell index fastest,
 * leading dimension `ld` >= ncells.  Element (species i, cell c) of VAR is
 * var[i*ld + c].  All batched arrays are DEVICE pointers; the small control
 * arrays ipar/rpar are HOST pointers.
 *
 * Return values of the entry points: KPP_B200_OK, or an error code below.
 * Integration failures are per cell, in IERR, with the reference's codes.
 */
#ifndef KPP_B200_H
#define KPP_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The entry points below are the library's only exported symbols: it is
   built with hidden visibility, so that the per-device set-up state of each
   mechanism library stays its own when several are loaded in one process. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define KPP_B200_OK 0
#define KPP_B200_EINVAL 1 /* invalid argument: size, null pointer, ld < ncells */
#define KPP_B200_ECUDA 2  /* CUDA runtime or launch error (see last_error) */

/* Per-cell integrator status codes (IERR), int/rosenbrock.c:186-199. */
#define KPP_B200_IERR_SUCCESS 1
#define KPP_B200_IERR_MAXSTEPS_BAD (-1)   /* improper value for max no of steps */
#define KPP_B200_IERR_METHOD (-2)         /* Rosenbrock method not implemented */
#define KPP_B200_IERR_HBOUNDS (-3)        /* Hmin/Hmax/Hstart must be positive */
#define KPP_B200_IERR_FACTORS (-4)        /* FacMin/FacMax/FacRej must be positive */
#define KPP_B200_IERR_TOLERANCES (-5)     /* improper tolerance values */
#define KPP_B200_IERR_TOO_MANY_STEPS (-6) /* no of steps exceeds maximum bound */
#define KPP_B200_IERR_STEP_TOO_SMALL (-7) /* step size too small */
#define KPP_B200_IERR_SINGULAR (-8)       /* matrix is repeatedly singular */

/* Mechanism description.
 * dims[0..5] = NVAR, NFIX, NSPEC, NREACT, LU_NONZERO, NONZERO.
 * Replaces the constants of the generated KPP_ROOT_Parameters.h
 * (src/gen.c:2627-2720). */
int kpp_b200_dims(int *dims);
const char *kpp_b200_mechanism_name(void);
/* SPC_NAMES[i] of the generated KPP_ROOT_Monitor.c; "" outside [0,NSPEC). */
const char *kpp_b200_species_name(int i);
/* C[0..NSPEC) after the generated Initialize() (values of #INITVALUES times
 * CFACTOR, src/gen.c:3172-3290) and the mechanism's CFACTOR. */
int kpp_b200_initial_values(double *c, double *cfactor);
/* LU_IROW/LU_ICOL [LU_NONZERO] and LU_CROW/LU_DIAG [NVAR+1] of the
 * generated KPP_ROOT_JacobianSP.c (src/gen.c:530-586). */
int kpp_b200_lu_pattern(int *irow, int *icol, int *crow, int *diag);

/* Batched Rosenbrock integration -- the drop-in for the generated INTEGRATE
 * path: for each cell c in [0, ncells), the same computation as
 *   Rosenbrock(VAR_c, tstart[c], tend[c], ATOL, RTOL, FunTemplate,
 *              JacTemplate, RPAR, IPAR)            (int/rosenbrock.c:137)
 * with the generator globals of that cell (FIX, TEMP, CFACTOR, SUN) taken
 * from the batched inputs.  Replaces the per-cell INTEGRATE calls of
 * drv/general.c:59-76 (int/rosenbrock.c:94-133).
 *
 *   var      [NVAR][ld]  in/out   VAR of every cell
 *   fix      [NFIX][ld]  in       FIX of every cell (may be NULL if NFIX == 0)
 *   temp     [ld]        in       TEMP
 *   cfactor  [ld]|NULL   in       CFACTOR (NULL: the mechanism's CFACTOR)
 *   sun      [ld]|NULL   in       SUN held constant over the call (NULL: SUN
 *                                 from Update_SUN(TIME) at every evaluation)
 *   tstart, tend [ld]    in       integration interval of each cell
 *   atol, rtol           in       device arrays, [NVAR] when ipar[1] == 0,
 *                                 else [1] (scalar tolerances)
 *   ipar [20], rpar[20]  in       HOST arrays, the integrator controls with
 *                                 the C indexing of int/rosenbrock.c:201-254:
 *                                 ipar[0] autonomous, ipar[1] scalar tol,
 *                                 ipar[2] max steps, ipar[3] method (1 Ros2,
 *                                 2 Ros3, 3 Ros4, 4 Rodas3, 5 Rodas4);
 *                                 rpar[0..6] Hmin, Hmax, Hstart, FacMin,
 *                                 FacMax, FacRej, FacSafe.  Entries 10..19
 *                                 are ignored (statistics start at zero).
 *   hstart   [ld]|NULL   in       per-cell starting step, replaces rpar[2]
 *                                 (warm start from the previous call's Hexit)
 *   istatus  [8][ld]     out      IPAR[10..17]: Nfun, Njac, Nstp, Nacc, Nrej,
 *                                 Ndec, Nsol, Nsng
 *   rstatus  [2][ld]     out      RPAR[10..11]: Texit, Hexit
 *   ierr     [ld]        out      return value of Rosenbrock for the cell
 *   stream               in       cudaStream_t, asynchronous
 */
int kpp_b200_rosenbrock(int ncells, int ld, double *var, const double *fix,
                        const double *temp, const double *cfactor,
                        const double *sun, const double *tstart,
                        const double *tend, const double *atol,
                        const double *rtol, const int *ipar,
                        const double *rpar, const double *hstart,
                        int *istatus, double *rstatus, int *ierr,
                        void *stream);

/* The reference's C SDIRK integrator (int/sdirk.c: SDIRK(N, Tinitial,
 * Tfinal, Y, RelTol, AbsTol, RCNTRL, ICNTRL, RSTATUS, ISTATUS),
 * int/sdirk.c:170-511) for every cell, on the same generated Fun / Jac_SP /
 * LU / solve as the Rosenbrock entries.  icntrl[20] / rcntrl[20] are the C
 * ICNTRL / RCNTRL: icntrl[1] = 0 vector tolerances, icntrl[2] the method (1
 * Sdirk2a, 2 Sdirk2b, 3 Sdirk3a, 4 Sdirk4a, 5 Sdirk4b, others Sdirk2a),
 * icntrl[3] the step limit, icntrl[4] the Newton limit, icntrl[5] = 1 zero
 * Newton start; rcntrl[0..10] Hmin, Hmax, Hstart, FacMin, FacMax, FacRej,
 * FacSafe, ThetaMin, NewtonTol, Qmin, Qmax.  Outputs follow the reference's
 * Fortran-style slots: istatus[8][ld] = ISTATUS[1..8] (Nfun, Njac, Nstp,
 * Nacc, Nrej, Ndec, Nsol, Nsng of this call), rstatus[3][ld] = RSTATUS[1..3]
 * (Texit, Hexit, Hnew, set at accepted steps, 0 before), ierr[ld] = the
 * reference's return value: 1 on success and 0 when it gave up (too many
 * steps, step too small) -- its error codes are printed, not returned.
 * Device pointers, asynchronous. */
int kpp_b200_sdirk(int ncells, int ld, double *var, const double *fix,
                   const double *temp, const double *cfactor, const double *sun,
                   const double *tstart, const double *tend, const double *atol,
                   const double *rtol, const int *icntrl, const double *rcntrl,
                   int *istatus, double *rstatus, int *ierr, void *stream);

/* The reference's C fully implicit Runge-Kutta integrator (int/runge_kutta.c:
 * RungeKutta(N, T, Tend, Y, RelTol, AbsTol, RCNTRL, ICNTRL, RSTATUS, ISTATUS,
 * &IERR), int/runge_kutta.c:203-1001) for every cell, with the complex LU of
 * util/sutil.c:28-90 generated for the mechanism.  icntrl[20] / rcntrl[20]
 * are the C ICNTRL / RCNTRL: icntrl[1] = 0 vector tolerances, icntrl[2] the
 * method (0 or 1 Radau-2A, 2 Lobatto-3C, 3 Gauss, 4 Radau-1A, 5 Lobatto-3A),
 * icntrl[3] the step limit, icntrl[4] the Newton limit, icntrl[5] = 1 zero
 * Newton start, icntrl[9] = 1 the SDIRK error estimator (0 the classic one),
 * icntrl[10] = 1 the classic step controller (0 Gustafsson's);
 * rcntrl[0..10] Hmin, Hmax, Hstart, FacMin, FacMax, FacRej, FacSafe,
 * ThetaMin, NewtonTol, Qmin, Qmax.  Outputs: istatus[8][ld] = ISTATUS[0..7]
 * (Nfun, Njac, Nstp, Nacc, Nrej, Ndec, Nsol, Nsng, counted as the reference
 * counts them), rstatus[3][ld] = RSTATUS[0..2] (Texit, Hacc, Hnew), ierr[ld]
 * = IERR: 1, or the last failing parameter check (-1, -2, -4 .. -8, -13) with
 * no step taken.  The reference prints the errors it meets while integrating
 * and carries on; here a cell whose step size becomes 0 or NaN stops with
 * -10 and one that needs more than icntrl[3] + 200000 steps with -9 (the
 * reference would not return from either).  Device pointers,
 * asynchronous. */
int kpp_b200_runge_kutta(int ncells, int ld, double *var, const double *fix,
                         const double *temp, const double *cfactor, const double *sun,
                         const double *tstart, const double *tend, const double *atol,
                         const double *rtol, const int *icntrl, const double *rcntrl,
                         int *istatus, double *rstatus, int *ierr, void *stream);

/* kpp_b200_sdirk and kpp_b200_runge_kutta on HOST arrays, for a host model
 * that keeps its cells in host memory as the reference's INTEGRATE does
 * (int/sdirk.c:92-166, int/runge_kutta.c:114-198): chunks of `chunk` cells
 * (0: 2^18) are copied in, integrated and copied back on two alternating
 * streams, so copies overlap the integration; synchronous.  Same arguments
 * and results as the device entries; pinned host memory gives full overlap. */
int kpp_b200_sdirk_host(int ncells, int ld, double *var, const double *fix,
                        const double *temp, const double *cfactor, const double *sun,
                        const double *tstart, const double *tend, const double *atol,
                        const double *rtol, const int *icntrl, const double *rcntrl,
                        int *istatus, double *rstatus, int *ierr, int chunk);
int kpp_b200_runge_kutta_host(int ncells, int ld, double *var, const double *fix,
                              const double *temp, const double *cfactor, const double *sun,
                              const double *tstart, const double *tend, const double *atol,
                              const double *rtol, const int *icntrl, const double *rcntrl,
                              int *istatus, double *rstatus, int *ierr, int chunk);

/* The Rosenbrock discrete adjoint, RosenbrockADJ (int/rosenbrock_adj.c:191-597)
 * per cell, replacing the model's INTEGRATE_ADJ loop over cells
 * (drv/general_adj.c): a forward Rosenbrock integration of var from tstart[c]
 * to tend[c] that keeps each accepted step (T, H, stage states, stage
 * vectors, and the factorised matrix when ICNTRL[7] != 0) in the cell's
 * trajectory, then the backward pass over it that updates the nadj adjoint
 * vectors in lambda[nadj * NVAR][ld] (adjoint m's entry i in row
 * m * NVAR + i) in place.  ICNTRL / RCNTRL in the C layout of
 * int/rosenbrock_adj.c (method ICNTRL[2]: 0/4 Rodas3, 1 Ros2, 2 Ros3, 3 Ros4,
 * 5 Rodas4, 7 Rodas3_1; ICNTRL[6]: 0/2 discrete adjoint, 1 forward only; 3
 * and 4, the continuous adjoints, are not built: EINVAL).  bufsize is the
 * trajectory capacity per cell, the reference's `bufsize` global: the step
 * limit is bufsize - 1, and any ICNTRL[3] != 0 returns IERR -1, as in the
 * reference.  work: a device buffer of at least
 * kpp_b200_rosenbrock_adj_work_bytes(ld, nadj, bufsize, ICNTRL[7]) bytes.
 * Outputs: istatus[8][ld] = ISTATUS[1..8] (forward and backward counters),
 * rstatus[3][ld] = Texit, Hexit, Hnew; ierr[ld].  Only in the libraries
 * built on KPP's own generator with the Hessian
 * (libkpp_b200_<mech>_kpproute.so); elsewhere EINVAL.  Asynchronous on
 * `stream`.  No single counterpart: the batched form of RosenbrockADJ. */
size_t kpp_b200_rosenbrock_adj_work_bytes(int ld, int nadj, int bufsize, int save_lu);
int kpp_b200_rosenbrock_adj(int ncells, int ld, double *var, const double *fix,
                            const double *temp, const double *cfactor, const double *sun,
                            const double *tstart, const double *tend, const double *atol,
                            const double *rtol, int nadj, double *lambda, const int *icntrl,
                            const double *rcntrl, int bufsize, double *work, size_t work_bytes,
                            int *istatus, double *rstatus, int *ierr, void *stream);

/* The host model's time loop (drv/general.c:59-76) over INTEGRATE
 * (int/rosenbrock.c:94-133) for every cell in one persistent launch: each cell
 * makes ncalls consecutive calls Rosenbrock(T, T + dt) with T = tstart[c]
 * first and T += dt after each call; the first call's Hstart is hstart[c]
 * (RPAR[2] when hstart is NULL), every later call's Hstart is the previous
 * call's Hexit (INTEGRATE's STEPMIN = RPAR[11]).  A failing call does not
 * stop the cell (the reference driver goes on after INTEGRATE reports it).
 * Outputs: var after the last call; istatus[8][ld] summed over the calls
 * (as INTEGRATE sums Ns/Na/Nr/Ng); rstatus[2][ld] Texit/Hexit of the last
 * call; ierr[ld] the first failing call's IERR, 1 when all succeed.
 * Equal, bit for bit, to ncalls kpp_b200_rosenbrock calls chained that way.
 * Cells are handed to warps through a device work queue, 32 at a time, in
 * the order order[0..ncells-1] (a permutation of 0..ncells-1; NULL for
 * 0,1,...); per-cell results do not depend on the order, the run time does:
 * the cost-binning scheduler passes cells sorted by decreasing predicted
 * cost.  Device pointers, asynchronous; the first call per (device, stream)
 * allocates the workspace and queue counter, so make it before capturing
 * the stream into a CUDA graph.  Uses the thread-per-cell kernel. */
int kpp_b200_rosenbrock_chain(int ncells, int ld, double *var,
                              const double *fix, const double *temp,
                              const double *cfactor, const double *sun,
                              const double *tstart, double dt, int ncalls,
                              const double *atol, const double *rtol,
                              const int *ipar, const double *rpar,
                              const double *hstart, const int *order,
                              int *istatus, double *rstatus, int *ierr,
                              void *stream);

/* Device workspace (bytes) that kpp_b200_rosenbrock_ws uses at most for a
 * batch of ncells cells; 0 for mechanisms whose work arrays fit in registers.
 * No counterpart in the reference (its integrator keeps its work arrays on
 * the host stack, int/rosenbrock.c:470-476). */
size_t kpp_b200_workspace_bytes(int ncells);

/* kpp_b200_rosenbrock with a caller-owned device workspace instead of the
 * library's cached one (for callers that manage device memory themselves or
 * run concurrent batches on one stream).  A workspace smaller than
 * kpp_b200_workspace_bytes(ncells) is rejected with KPP_B200_EINVAL. */
int kpp_b200_rosenbrock_ws(int ncells, int ld, double *var, const double *fix,
                           const double *temp, const double *cfactor,
                           const double *sun, const double *tstart,
                           const double *tend, const double *atol,
                           const double *rtol, const int *ipar,
                           const double *rpar, const double *hstart,
                           int *istatus, double *rstatus, int *ierr,
                           void *workspace, size_t workspace_bytes,
                           void *stream);

/* Allocation-free kpp_b200_rosenbrock.  No counterpart in the reference.
 * For callers that cannot allocate device memory -- code running where
 * cudaMalloc is not allowed (inside a stream capture that must not allocate,
 * a host model with a fixed device-memory budget, or a library that is handed
 * only its inputs and outputs).  The caller still passes every input and
 * output; the work arrays live in a fixed device array inside the library,
 * sized for at most 1024 cells per call (about 21 MB for saprc99; 128 cells,
 * 22 MB, for mechanisms whose per-cell work arrays would make 1024 cells
 * exceed 64 MB, such as MCM isoprene), reserved on every GPU that loads the
 * library, until exit.  Larger batches are rejected with KPP_B200_EINVAL;
 * split them into calls of at most that many cells.
 * The first call on a device looks up that array's device address, so make it
 * before any stream capture.  No memory is allocated or freed by any call.
 * Every call uses the same array: calls that overlap on the GPU (concurrent
 * streams) race on it, so issue them on one stream or serialise them.  No
 * state carries over between calls: each call writes every work element
 * before reading it, so nothing needs clearing. */
int kpp_b200_rosenbrock_static(int ncells, int ld, double *var, const double *fix,
                               const double *temp, const double *cfactor,
                               const double *sun, const double *tstart,
                               const double *tend, const double *atol,
                               const double *rtol, const int *ipar,
                               const double *rpar, const double *hstart,
                               int *istatus, double *rstatus, int *ierr,
                               void *stream);

/* kpp_b200_rosenbrock on HOST arrays (same layout and meaning, all batched
 * arrays in host memory, pinned for full copy/compute overlap): the batch is
 * cut into chunks of `chunk` cells (0: library default) that go through
 * host->device copy, integration and device->host copy on two streams, so the
 * copies of one chunk overlap the integration of the other.  var, istatus,
 * rstatus and ierr are written back to the host arrays.  Synchronous: returns
 * when every output is in host memory.  This is the drop-in for a host model
 * that keeps its grid in host memory and calls INTEGRATE for every cell
 * (drv/general.c:59-76). */
int kpp_b200_rosenbrock_host(int ncells, int ld, double *var, const double *fix,
                             const double *temp, const double *cfactor,
                             const double *sun, const double *tstart,
                             const double *tend, const double *atol,
                             const double *rtol, const int *ipar,
                             const double *rpar, const double *hstart,
                             int *istatus, double *rstatus, int *ierr,
                             int chunk);

/* Batched evaluation of the generated mechanism functions at time `time`
 * (the same for all cells), each exactly as FunTemplate / JacTemplate /
 * Update_RCONST compute it (int/rosenbrock.c:1257-1296, src/gen.c:642-724,
 * 1185-1322, 2343-2473).  Any of rconst [NREACT][ld], vdot [NVAR][ld],
 * jvs [LU_NONZERO][ld] may be NULL.  Device pointers, asynchronous. */
int kpp_b200_fun_jac(int ncells, int ld, const double *var, const double *fix,
                     const double *temp, const double *cfactor,
                     const double *sun, double time, double *rconst,
                     double *vdot, double *jvs, void *stream);

/* The building blocks of the discrete adjoint (int/rosenbrock_adj.c), for
 * every cell: out = J uv (transposed = 0, Jac_SP_Vec) or out = J^T uv
 * (transposed = 1, JacTR_SP_Vec), src/gen.c:1763-1880, with jvs
 * [LU_NONZERO][ld] in the LU pattern, uv and out [NVAR][ld] (out must not be
 * uv); and the solve of (LU)^T xx = x for a factorised jvs (KppSolveTR,
 * src/gen.c:2036-2120; xx may be x).  Same operations in the same order as
 * the generated C functions.  Device pointers, asynchronous. */
int kpp_b200_jac_vec(int ncells, int ld, const double *jvs, const double *uv,
                     double *out, int transposed, void *stream);
int kpp_b200_solve_tr(int ncells, int ld, const double *jvs, const double *x,
                      double *xx, void *stream);

/* Batched no-pivot sparse LU (KppDecomp, util/sutil.c:2-23) of jvs
 * [LU_NONZERO][ld] in place, then one solve (KppSolve, src/gen.c:1960-2034)
 * of x [NVAR][ld] in place when x is not NULL.  ising[ld] receives the
 * KppDecomp return value.  Device pointers, asynchronous. */
int kpp_b200_decomp_solve(int ncells, int ld, double *jvs, double *x,
                          int *ising, void *stream);

/* Kernel used by the Rosenbrock entries (process-wide): 0 automatic (the
 * default), 1 one thread per cell with the work set in device memory, 2 one
 * warp per cell with the work set in shared memory (the mechanism's schedule
 * tables staged in shared memory once per CTA; no work buffer).  Kernel 2 runs
 * the launches whose rate constants are fixed for the call (SUN given per
 * cell, or no SUN-dependent rates; no rates of time or concentrations) of
 * mechanisms with at most 1024 LU entries; other launches use kernel 1.  Both
 * kernels give bit-identical results.  Automatic selects kernel 2 for such
 * launches of at most kpp_b200_get_auto_warp_cells() cells (by default every
 * size for mechanisms with a per-cell work buffer: on B200 with saprc99 it
 * measured faster from 2^11 to 2^20 cells), except single calls given a
 * per-cell Hstart (warm-started short calls, where the thread kernel measured
 * 4.7x faster), and kernel 1 otherwise.  No counterpart in the reference.
 * kpp_b200_get_kernel returns the configured kernel (1 or 2; 1 for
 * automatic). */
int kpp_b200_set_kernel(int which);
int kpp_b200_get_kernel(void);

/* Work-queue granularity of kpp_b200_rosenbrock_chain on the thread-per-cell
 * kernel (process-wide): 0 each warp takes the next 32 queue positions and
 * its lanes start every chained call together; 1 (the default) each lane
 * takes the next single position as soon as its previous cell is done, and
 * the lanes' cells advance together one step attempt at a time however far
 * apart they are, so no lane idles until the slowest cell of its warp
 * finishes.  Results do not depend on it.  No counterpart in the reference. */
int kpp_b200_set_queue_lanes(int per_lane);
int kpp_b200_get_queue_lanes(void);

/* The automatic choice's limit (process-wide): launches of at most `ncells`
 * cells use the warp-per-cell kernel when they can (0: never).  The autotuner
 * (kpp_b200/autotune.py) measures both kernels per device, mechanism and
 * workload.  No counterpart in the reference. */
int kpp_b200_set_auto_warp_cells(int ncells);
int kpp_b200_get_auto_warp_cells(void);

/* Launch shape of the thread-per-cell kernel (process-wide): the number of
 * 128-thread blocks per SM the Rosenbrock entries keep resident, 0 (the
 * default) for as many as fit.  Fewer resident cells thrash L2 less; the
 * autotuner (kpp_b200/autotune.py) picks the value per device and workload.
 * Results do not depend on it.  No counterpart in the reference. */
int kpp_b200_set_blocks_per_sm(int blocks);
int kpp_b200_get_blocks_per_sm(void);

/* Host-model species order (GenerateShuffle_user2kpp / _kpp2user,
 * src/gen.c:3401-3468): user species k is the k-th species the mechanism
 * declares as variable, unused ones included, among its first NSPEC - 1
 * declared species (the reference's loop bound); kpp_index[k] is its index
 * in the library's VAR order, or -1 when it takes no part in the mechanism
 * (or k >= NVAR, where the reference's shuffle stops).  *nuser receives the
 * number of user species; either pointer may be NULL. */
int kpp_b200_user_species(int *nuser, int *kpp_index);

/* Batched Shuffle_user2kpp: var[kpp_index[k]][c] = v_user[k][c] for every
 * mapped user species k (v_user [nuser][ld_user], var [NVAR][ld], cell index
 * fastest); other VAR rows are left as they are.  Device pointers,
 * asynchronous. */
int kpp_b200_shuffle_user2kpp(int ncells, int ld_user, const double *v_user, int ld,
                              double *var, void *stream);

/* Batched Shuffle_kpp2user: v_user[k][c] = var[kpp_index[k]][c] for every
 * mapped user species k; unmapped rows of v_user are left as they are. */
int kpp_b200_shuffle_kpp2user(int ncells, int ld, const double *var, int ld_user,
                              double *v_user, void *stream);

/* Text of the last error of this thread's last failing call. */
const char *kpp_b200_last_error(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* KPP_B200_H */
