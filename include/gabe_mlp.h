/* gabe_mlp.h -- spectra emulator: a small MLP trained and queried on the GPU.
 *
 * No counterpart in the reference (GABE runs lattices only).  The network
 * maps (log g^2/lambda, amplitude multiplier, time) to the ensemble's binned
 * log spectra (gabe_ensemble_log_spectra: 3 x nlog values).  Layout:
 *
 *   n_in -> width (SiLU) -> ... depth hidden layers ... -> n_out (linear)
 *
 * Weights, biases, gradients and Adam moments are FP32; activations between
 * layers are stored in BF16 (GABE_MLP_FP32_ACT stores them in FP32); every
 * product is accumulated in FP32.  The forward of a BF16 layer whose BF16
 * weights fit in shared memory (K <= 256, N <= 256, K a multiple of 64, N
 * of 32) runs on the fifth-generation tensor cores (tcgen05, TMEM
 * accumulators), other BF16 layers on mma.sync, the first layer and the
 * backward products on FP32 FMA.  Flat parameter layout, layer by layer:
 * W_l [K_l][N_l] (row-major, K_l inputs) followed by b_l [N_l].
 *
 * Targets may hold NaN (log bins with no native bin): the loss is the mean
 * of (y - t)^2 over the finite targets only.
 *
 * All data pointers are DEVICE pointers unless named h_*; every call is
 * asynchronous on the handle's stream except those returning host data.
 * ------------------------------------------------------------------------ */
#ifndef GABE_MLP_H
#define GABE_MLP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GABE_MLP_FP32_ACT 1   /* store activations in FP32 instead of BF16 */
#define GABE_MLP_NO_GRAPH 2   /* launch training steps directly (no CUDA graph) */
#define GABE_MLP_MMA_SYNC 4   /* forward of the BF16 layers on the mma.sync kernel instead of tcgen05 */

typedef struct {
    int32_t struct_size;   /* sizeof(gabe_mlp_params) */
    int32_t n_in;          /* inputs (3) */
    int32_t width;         /* hidden width (256), multiple of 64 */
    int32_t depth;         /* hidden layers (4) */
    int32_t n_out;         /* outputs (3 x 64 = 192), multiple of 64 */
    int32_t max_rows;      /* largest batch a forward/training call handles at once */
    float lr, beta1, beta2, eps, weight_decay;  /* AdamW */
    float lr_min;          /* cosine decay of the learning rate from lr to lr_min ... */
    int32_t decay_steps;   /* ... over this many Adam steps (0 = constant lr) */
    uint64_t seed;         /* weight initialisation */
    int32_t device;        /* CUDA device, -1 = current */
    int32_t flags;         /* GABE_MLP_* */
} gabe_mlp_params;

typedef struct gabe_mlp gabe_mlp;

void gabe_mlp_default_params(gabe_mlp_params *p);
int gabe_mlp_create(const gabe_mlp_params *p, gabe_mlp **out);
int gabe_mlp_destroy(gabe_mlp *m);
int64_t gabe_mlp_num_params(const gabe_mlp *m);

/* Copy all parameters (flat layout above) from / to host memory. */
int gabe_mlp_set_params(gabe_mlp *m, const float *h_params);
int gabe_mlp_get_params(gabe_mlp *m, float *h_params);

/* y [n][n_out] = net(x [n][n_in]); any n >= 0 (processed in chunks of max_rows). */
int gabe_mlp_forward(gabe_mlp *m, const float *x, int64_t n, float *y);

/* Loss and gradient of one batch (n <= max_rows), for checks: h_loss = mean
 * squared error over finite targets; h_grad (may be NULL) = d loss / d
 * params in the flat layout.  Parameters are not changed. */
int gabe_mlp_loss_grad(gabe_mlp *m, const float *x, const float *t, int64_t n, double *h_loss, float *h_grad);

/* nbatch AdamW steps: step s trains on rows perm[(s0 + s) * batch + i],
 * i < batch, of x [*][n_in] and t [*][n_out], where s0 counts the batches
 * taken since the last gabe_mlp_reset_batches.  The caller keeps perm
 * valid for (s0 + nbatch) * batch entries. */
/* Learning-rate schedule for the following Adam steps: cosine from lr to
 * lr_min over decay_steps steps counted from the first step taken (0 =
 * constant lr). */
int gabe_mlp_set_schedule(gabe_mlp *m, float lr, float lr_min, int32_t decay_steps);

int gabe_mlp_train(gabe_mlp *m, const float *x, const float *t, const int32_t *perm, int32_t batch, int32_t nbatch);
int gabe_mlp_reset_batches(gabe_mlp *m);

/* Mean of the batch losses since the last call (reads back; syncs), and the
 * number of Adam steps taken so far. */
int gabe_mlp_train_loss(gabe_mlp *m, double *h_mean_loss, int64_t *h_steps);

/* Waits for the handle's stream; GABE_ERR_TIMEOUT if a bounded device wait
 * of the tensor-core forward gave up since the handle was created. */
int gabe_mlp_sync(gabe_mlp *m);
/* Kernel that runs the forward of layer `layer`: 0 FP32 FMA, 1 mma.sync,
 * 2 tcgen05; -1 for a bad layer index. */
int gabe_mlp_forward_form(const gabe_mlp *m, int32_t layer);
void *gabe_mlp_stream(const gabe_mlp *m);
/* The library's kernel launches per training step and per forward chunk. */
int gabe_mlp_launches_per_train_step(const gabe_mlp *m);
int gabe_mlp_launches_per_forward(const gabe_mlp *m);
const char *gabe_mlp_last_error(const gabe_mlp *m);

#ifdef __cplusplus
}
#endif
#endif
