/* Learned warm start for the lane sweep: C ABI.
 *
 * No counterpart in the reference. ESPice starts a sweep point's Newton from
 * the nominal operating point (`--warm-start`, src/analysis/dc/op.zig
 * coldStart / the points API's warm start); this module predicts a start point
 * per lane from the lane's sweep parameters with a small MLP
 * (in -> 128 -> 128 -> out, tanh hidden layers) whose dense layers run on the
 * B200 tensor cores (tcgen05, BF16 operands, FP32 accumulation). It is trained
 * on operating points the plain method produced; the converged answer is
 * still the plain Newton's (espl_solve_static from the predicted x), so only
 * the iteration count changes.
 *
 * Arrays are host memory, row-major, one row per lane; a call borrows them
 * only while it runs. Status codes are espice_lanes.h's.
 */
#ifndef ESPICE_LEARNED_H
#define ESPICE_LEARNED_H

#include <stddef.h>
#include <stdint.h>

#include "espice_lanes.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct espl_mlp espl_mlp;

typedef struct {
    uint32_t epochs;
    uint32_t batch;     /* rows per Adam step (<= the capacity) */
    float lr;           /* Adam step size at the first epoch */
    float lr_final;     /* > 0: geometric decay to this at the last epoch */
    float beta1, beta2, eps;
    uint32_t seed;      /* minibatch shuffling */
} espl_train_opts;

/* A network for `in_dim` parameters and `out_dim` unknowns (both <= 128),
 * with device buffers for batches of up to `capacity` rows, weights drawn
 * from `seed` (Glorot uniform, zero biases). */
espl_status espl_mlp_create(uint32_t in_dim, uint32_t out_dim, uint32_t capacity, uint64_t seed, uint32_t device,
                            espl_mlp **out);
espl_status espl_mlp_destroy(espl_mlp *m);

/* Parameters in the order W1 [128 x in], b1 [128], W2 [128 x 128], b2 [128],
 * W3 [out x 128], b3 [out], row-major, FP32 (the master copy; the GEMMs read
 * its BF16 rounding). */
espl_status espl_mlp_param_count(const espl_mlp *m, uint32_t *count);
espl_status espl_mlp_get_params(espl_mlp *m, float *params);
espl_status espl_mlp_set_params(espl_mlp *m, const float *params);

/* Per-feature standardization of inputs and targets from a data set (mean
 * and population standard deviation; a constant feature keeps scale 1).
 * espl_mlp_train sets it from its data when it was never set. */
espl_status espl_mlp_set_scaling(espl_mlp *m, const double *x, const double *y, uint32_t n);

/* One forward + backward pass over n <= capacity rows: the mean squared error
 * of the standardized outputs and its gradient in espl_mlp_get_params order.
 * The weights are not changed. */
espl_status espl_mlp_loss_grad(espl_mlp *m, const double *x, const double *y, uint32_t n, double *loss,
                               float *grad);

/* Adam over minibatches of a shuffled data set; epoch_loss (optional) gets
 * the mean minibatch loss of every epoch. */
espl_status espl_mlp_train(espl_mlp *m, const double *x, const double *y, uint32_t n, const espl_train_opts *opts,
                           double *epoch_loss);

/* The same from a data set already in device memory (x: n x in_dim, y:
 * n x out_dim, FP64, row-major, device pointers, e.g. the transient's
 * recorded steps from espl_recorded_steps): the standardization, when never
 * set, is computed on the device. */
espl_status espl_mlp_train_device(espl_mlp *m, const double *x, const double *y, uint32_t n,
                                  const espl_train_opts *opts, double *epoch_loss);

/* Device time of the last training call (CUDA events on the network's
 * stream around its standardization and Adam steps; allocations and host
 * copies excluded), milliseconds. */
espl_status espl_mlp_train_ms(const espl_mlp *m, double *device_ms);
/* Device time of the last espl_mlp_predict (CUDA events on the network's
 * stream around its copies and its launch), milliseconds. */
espl_status espl_mlp_predict_ms(const espl_mlp *m, double *device_ms);

/* Predictions for n rows (any n): one fused inference launch, each CTA
 * running the whole network on 128 rows from shared memory and tensor
 * memory. */
espl_status espl_mlp_predict(espl_mlp *m, const double *x, uint32_t n, double *y);
/* The same predictions layer by layer through the training GEMMs, in
 * capacity-sized chunks (a cross-check of the fused kernel). */
espl_status espl_mlp_predict_layers(espl_mlp *m, const double *x, uint32_t n, double *y);

espl_status espl_mlp_error_message(espl_mlp *m, char *buf, size_t cap);

/* ---- The learned next-step predictor of the transient lanes ----
 *
 * Replaces the reference's linear predictor x = cur + (dt / dt_old)
 * (cur - prev) (src/solver/lane_device.zig:388, src/solver/kernels/lane.zig
 * :473-482) as the Newton start of a transient attempt, for the lanes of
 * the templates that have a network attached, when espl_tran_opts.predictor
 * is 2. The network's input is the lane's last three accepted solutions and
 * the step about to be taken, as D = 3 n + 1 features:
 *   f[i]        = cur[i]
 *   f[n + i]    = (dt / h0) (cur[i] - prev[i])
 *   f[2 n + i]  = (dt / h1) (prev[i] - prev2[i])
 *   f[3 n]      = dt / dt_max
 * (cur, prev, prev2 the solutions at the last three accepted steps, h0 and h1
 * the last two accepted step sizes, dt the step attempted); its output is
 * the correction to the linear predictor, x_start = cur + (dt / h0)
 * (cur - prev) + y. Before the lane's fourth accepted step the linear
 * predictor stands. The plain Newton stays judge and fallback: an attempt
 * that does not converge from the learned start is retried once at the same
 * step from the linear predictor (not counted as a rejected step), so the
 * accepted steps are the plain method's; with espl_create_opts.polish the
 * converged points do not depend on the start to well below the Newton
 * tolerance. Attempts of lanes with a network run one per launch (a CUDA
 * graph of the predictor kernel and one attempt, replayed), the other
 * templates' lanes in one persistent launch as with the other predictors. */

/* Records, from the next accepted steps on, the training samples of
 * template `net`: lanes l with l % lane_stride == 0, accepted steps past
 * `from_step`, at most `capacity` samples (FP64, on the device): features as
 * above and target y = x_accepted - (cur + (dt / h0) (cur - prev)). Calling
 * it again restarts the recording; capacity 0 stops it. */
espl_status espl_record_steps(espl_lanes *h, uint32_t net, uint32_t lane_stride, uint32_t from_step,
                              uint32_t capacity);
/* The recorded samples: *x (count x (3 n + 1)) and *y (count x n) are
 * DEVICE pointers owned by the handle (valid until the next
 * espl_record_steps or destroy), *count the samples kept. */
espl_status espl_recorded_steps(espl_lanes *h, uint32_t net, const double **x, const double **y, uint32_t *count);
/* Host copies of the first min(count, cap) recorded samples: x (3 n + 1 per
 * sample), y (n), tags (5: the lane, its accepted steps before this one, dt,
 * h0, h1); any may be NULL. */
espl_status espl_copy_recorded_steps(espl_lanes *h, uint32_t net, double *x, double *y, double *tags, uint32_t cap);
/* Attaches network m (in_dim 3 n + 1, out_dim n of template `net`) as the
 * template's step predictor (NULL detaches). The network is borrowed: it
 * must outlive its use; retraining it takes effect at the next launch. */
espl_status espl_set_step_predictor(espl_lanes *h, uint32_t net, espl_mlp *m);
/* Runs the step predictor of template `net` on the lanes' current state and
 * copies out the learned start of each lane's next attempt (x_start,
 * [lanes][n], host; NaN rows where a lane has no learned start yet), with
 * the history it read: cur, prev, prev2 ([lanes][n]) and steps (dt, h0, h1
 * per lane, [lanes][3]); any output may be NULL. */
espl_status espl_step_predict(espl_lanes *h, uint32_t net, double *x_start, double *cur, double *prev, double *prev2,
                              double *steps);

#ifdef __cplusplus
}
#endif
#endif
