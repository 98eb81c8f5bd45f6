/* kpp_sched.h -- learned cell scheduler for the batched Rosenbrock entries.
 *
 * No counterpart in the reference: KPP integrates one cell at a time
 * (drv/general.c:59-76) and starts every call at Hstart = STEPMIN
 * (int/rosenbrock.c:102-104).  This library adds a small MLP that, from a
 * cell's state, proposes the starting step Hstart (RPAR[2] of the call) and
 * predicts the call's internal step count; the predicted cost sorts the cells
 * into the work-queue order of kpp_b200_rosenbrock_chain so that the 32 cells
 * of a warp cost about the same.  The Rosenbrock controller is unchanged and
 * still accepts or rejects every step.
 *
 * Network: nin inputs -> nhidden layers of `width` units with GELU (erf form)
 * -> nout outputs (log10 Hstart and ln Nstp, standardised).  Weights BF16 on
 * the tensor cores (mma.sync m16n8k16, FP32 accumulate), FP32 master copies,
 * FP32 biases; trained with Adam by the library's own kernels.
 *
 * Parameter layout (host and device, float): for each linear layer l in
 * order, W_l [out_l][in_l] row-major, then b_l [out_l].
 *
 * Features (kpp_sched_features), in this order: log10(max(VAR_i, 1e-20)) for
 * i < nvar, TEMP, ln CFACTOR, SUN (the per-cell value, or Update_SUN(TSTART)
 * when no per-cell SUN is given), ln(TEND - TSTART); standardised with the
 * model's input scaling.  Stored feature-major: x[f * ld_x + c] (cell index
 * fastest), BF16.
 *
 * All pointers are device pointers unless named host_*; every call is
 * asynchronous on `stream` (a cudaStream_t) and returns 0 or an error code.
 */
#ifndef KPP_SCHED_H
#define KPP_SCHED_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KPP_SCHED_OK 0
#define KPP_SCHED_EINVAL 1
#define KPP_SCHED_ECUDA 2

typedef struct kpp_sched_mlp kpp_sched_mlp;

/* Creates a network; buffers for training batches of up to max_batch rows
 * and for inference are allocated on the current device.  NULL on failure
 * (kpp_sched_last_error tells why). */
kpp_sched_mlp *kpp_sched_mlp_create(int nin, int width, int nhidden, int nout, int max_batch);
void kpp_sched_mlp_destroy(kpp_sched_mlp *m);
long kpp_sched_mlp_param_count(const kpp_sched_mlp *m);

/* Parameters (FP32, the layout above) in / out; set also refreshes the BF16
 * copies and resets the Adam state.  Synchronous. */
int kpp_sched_mlp_set_params(kpp_sched_mlp *m, const float *host_params);
int kpp_sched_mlp_get_params(const kpp_sched_mlp *m, float *host_params);
/* The BF16 weights the GEMMs use, as float (bias slots hold the FP32 bias). */
int kpp_sched_mlp_get_params_bf16(const kpp_sched_mlp *m, float *host_params);
/* Gradient of the last kpp_sched_mlp_loss_grad (FP32, parameter layout). */
int kpp_sched_mlp_get_grads(const kpp_sched_mlp *m, float *host_grads);

/* Standardisation: feature f -> (f - in_mu) / in_sd; output o -> o * out_sd
 * + out_mu.  Host arrays of nin and nout floats.  Synchronous. */
int kpp_sched_mlp_set_scaling(kpp_sched_mlp *m, const float *host_in_mu,
                              const float *host_in_sd, const float *host_out_mu,
                              const float *host_out_sd);

/* Forward pass of `batch` rows of x (feature-major, ld_x >= batch) into
 * out[batch][nout] (standardised outputs, FP32). */
int kpp_sched_mlp_forward(kpp_sched_mlp *m, int batch, const void *x_bf16, long ld_x,
                          float *out, void *stream);

/* Mean squared error of the network on (x, y) (y[batch][nout], standardised
 * targets) into *loss (device float), and its gradient into the library's
 * gradient buffer.  batch <= max_batch. */
int kpp_sched_mlp_loss_grad(kpp_sched_mlp *m, int batch, const void *x_bf16, long ld_x,
                            const float *y, float *loss, void *stream);

/* One Adam step (beta1, beta2, eps as given) with learning rate lr on the
 * last gradient; refreshes the BF16 weights. */
int kpp_sched_mlp_adam(kpp_sched_mlp *m, float lr, float beta1, float beta2, float eps,
                       void *stream);

/* Columns idx[0..n) of src (feature-major [nrows][ld_src]) into dst
 * ([nrows][ld_dst]): gathers a training minibatch. */
int kpp_sched_gather_columns(int nrows, int n, const int *idx, const void *src_bf16,
                             long ld_src, void *dst_bf16, long ld_dst, void *stream);

/* Features of ncells cells in the Rosenbrock ABI layout (var [nvar][ld],
 * temp/cfactor/sun/tstart/tend [ld]; cfactor, sun, tend may be NULL, tend
 * NULL means TEND - TSTART = dt) into x (feature-major, ld_x), standardised
 * with the model's scaling.  nin must be nvar + 4. */
int kpp_sched_features(const kpp_sched_mlp *m, int ncells, int ld, int nvar,
                       const double *var, const double *temp, const double *cfactor,
                       const double *sun, const double *tstart, const double *tend, double dt,
                       void *x_bf16, long ld_x, void *stream);

/* The scheduling pass over ncells cells: features, the network, and in the
 * output layer's epilogue Hstart = clamp(10^(log10 Hstart), hmin, hmax) and
 * the cost bin of the predicted ln Nstp (nbins bins over [lo, hi], most
 * expensive first); then a counting sort writes order[0..ncells) = the cells
 * by decreasing predicted cost (ties in any order).  pred (optional,
 * [ncells][nout]) receives the de-standardised outputs. */
int kpp_sched_plan(kpp_sched_mlp *m, int ncells, int ld, int nvar, const double *var,
                   const double *temp, const double *cfactor, const double *sun,
                   const double *tstart, const double *tend, double dt, double hmin,
                   double hmax, int nbins, float lnn_lo, float lnn_hi, double *hstart,
                   int *order, float *pred, void *stream);

const char *kpp_sched_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
