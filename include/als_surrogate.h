/* MLP surrogate of a scalar UQ observable, trained and evaluated with
 * hand-written BF16 tensor-core (tcgen05) kernels, FP32 accumulation.
 *
 * No counterpart in the reference: its Monte Carlo loop
 * (alsuq/src/run/Runner.cpp:42-78) and MeanVariance statistics
 * (alsuq/src/stats/MeanVariance.cpp:30-67) use plain sample averages.  The
 * surrogate maps the perturbation parameters of a sample (40 for
 * Kelvin-Helmholtz, drawn as in alsuq/src/generator/STLMersenne.cpp:38-85)
 * to the observable and serves as a control variate in the mean/variance
 * estimator.
 *
 * Network: inputs -> width (GELU) -> ... -> width (GELU) -> 1, `hidden`
 * hidden layers.  Parameters are one flat FP32 vector (master copy), layer
 * after layer, each layer's weight matrix (out x in, row-major) followed by
 * its bias; the tensor cores read BF16 copies of the weight matrices.
 * Activations between layers are BF16, pre-activations FP32.
 *
 * Pointers named *_dev are device pointers; all other arrays are host
 * memory.  Every function returns ALS_OK or a negative ALS_E* code, with
 * als_last_error() describing the failure.  Functions taking a stream
 * enqueue on it and return after the work has completed.  A handle's calls
 * share its device workspace: use a handle from one host thread at a time
 * (separate handles are independent).
 */
#ifndef ALS_SURROGATE_H
#define ALS_SURROGATE_H

#include "als_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct als_mlp als_mlp;

typedef struct {
    int inputs;       /* input features, 1..64 */
    int width;        /* hidden width: 64, 128 or 256 */
    int hidden;       /* hidden layers, 1..6 */
    int max_batch;    /* largest training / gradient batch, a multiple of 128 */
} als_mlp_config;

int als_mlp_create(const als_mlp_config* cfg, int device, als_mlp** out);
int als_mlp_destroy(als_mlp* h);

/* Number of parameters (208,129 for 40 -> 256 x4 -> 1). */
int als_mlp_param_count(const als_mlp* h, long long* count);

/* Deterministic initialisation from `seed` (weights and biases uniform in
 * +-1/sqrt(fan_in)); clears the Adam moments and step counter. */
int als_mlp_init(als_mlp* h, unsigned long long seed);

/* Copy the flat FP32 parameter vector in or out (host memory).  Setting
 * parameters refreshes the BF16 copies and clears the Adam state. */
int als_mlp_set_params(als_mlp* h, const float* params);
int als_mlp_get_params(const als_mlp* h, float* params);

/* Inference: y_dev[r] = f(x_dev[r, :]) for `rows` rows of `inputs` FP32
 * features (row-major).  Any number of rows.  Per 262,144 rows a 256-wide
 * network runs as two kernels: the inputs' BF16 rounding, then every layer
 * and the head in one kernel with the activations kept on the SM; other
 * widths run one kernel per layer. */
int als_mlp_forward(als_mlp* h, const float* x_dev, long long rows, float* y_dev, void* stream);

/* The same inference with one kernel per layer (activations through device
 * memory).  Its results equal als_mlp_forward's bit for bit. */
int als_mlp_forward_layers(als_mlp* h, const float* x_dev, long long rows, float* y_dev,
                           void* stream);

/* Gradient of the mean squared error (1/rows) sum (f(x_r) - t_r)^2 with
 * respect to the flat parameters, into grad_dev (param_count floats);
 * the loss into *loss (host).  rows <= max_batch. */
int als_mlp_gradients(als_mlp* h, const float* x_dev, const float* t_dev, int rows,
                      float* grad_dev, float* loss, void* stream);

/* `steps` full-batch Adam steps (beta1 0.9, beta2 0.999, eps 1e-8, learning
 * rate `lr`) on the mean squared error over `rows` samples, one CUDA graph
 * per step.  loss_dev (steps floats, or null) receives each step's loss. */
int als_mlp_train(als_mlp* h, const float* x_dev, const float* t_dev, int rows, int steps,
                  float lr, float* loss_dev, void* stream);

/* Failure-detection hook for tests.  Every wait of the tensor-core GEMMs
 * that compute gradients and train (and of inference when width is not
 * 256) polls its barrier at most `wait_limit` times (0: the default, about
 * 4 M polls) and, after a timeout, sets the handle's error flag, waits for
 * its own MMAs in flight, frees its tensor memory and returns; the call then
 * returns ALS_E_CUDA ("tensor-core GEMM wait timed out") and the handle and
 * the CUDA context stay usable.  With `withhold_commit` nonzero these GEMMs
 * issue no completion commit, so their waits run out (nothing else is
 * skipped); 0 restores normal operation. */
int als_mlp_test_wait_timeout(als_mlp* h, unsigned wait_limit, int withhold_commit);

/* U[0,1) draws (24-bit, counter based on `seed` and the index) into
 * x_dev[0 .. count). */
int als_mlp_sample_uniform(float* x_dev, long long count, unsigned long long seed, void* stream);

#ifdef __cplusplus
}
#endif

#endif
