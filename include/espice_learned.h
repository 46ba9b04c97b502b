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

/* Predictions for n rows (any n): one fused inference launch, each CTA
 * running the whole network on 128 rows from shared memory and tensor
 * memory. */
espl_status espl_mlp_predict(espl_mlp *m, const double *x, uint32_t n, double *y);
/* The same predictions layer by layer through the training GEMMs, in
 * capacity-sized chunks (a cross-check of the fused kernel). */
espl_status espl_mlp_predict_layers(espl_mlp *m, const double *x, uint32_t n, double *y);

espl_status espl_mlp_error_message(espl_mlp *m, char *buf, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
