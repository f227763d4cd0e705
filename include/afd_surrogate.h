/*
 * afd_surrogate.h - C ABI of the learned impulse-response surrogate and of
 * the BF16 tensor-core GEMM it is built on (sm_100a, tcgen05, FP32
 * accumulation). No counterpart in the reference: the reference has no
 * learned model. Training data come from the FDTD engine of afd.h, which
 * also serves as the fallback for predictions outside the error bound.
 *
 * Network: x (n_in values in [0, 1]) -> Fourier features
 * [sin(2 pi x B), cos(2 pi x B)] (B: n_in x n_freq drawn N(0, sigma^2) from
 * `seed`) -> (n_layers - 1) Linear+ReLU layers of `hidden` units -> Linear
 * to n_out values. Mean-squared-error loss, Adam. FP32 master weights with
 * BF16 copies for the GEMMs; activations and gradients in BF16.
 *
 * Sizes: 2*n_freq, hidden, n_out and batch multiples of 128.
 * Pointers x, y and out may be device or host memory (copied with
 * cudaMemcpyDefault); every call is synchronous unless noted.
 * Status codes are those of afd.h.
 */
#ifndef AFD_SURROGATE_H
#define AFD_SURROGATE_H

#include <stdint.h>

#include "afd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct afd_mlp afd_mlp;

typedef struct {
    int32_t n_in, n_freq, hidden, n_layers, n_out, batch, device;
    float fourier_sigma;
    uint64_t seed;
    float lr, beta1, beta2, eps;
    int32_t reserved[8];
} afd_mlp_params;

/* Tensors readable with afd_mlp_get. */
#define AFD_MLP_WEIGHT       0  /* layer weights [out][in] (FP32 master copy) */
#define AFD_MLP_BIAS         1  /* layer bias [out] */
#define AFD_MLP_GRAD_WEIGHT  2  /* gradient of the last train/gradients call */
#define AFD_MLP_GRAD_BIAS    3
#define AFD_MLP_FOURIER      4  /* B [n_in][n_freq] (layer ignored) */
#define AFD_MLP_FEATURES     5  /* BF16 features of the last call [batch][2*n_freq], as float */

/* 10 inputs, 128 frequencies, 5 layers of 512 hidden units, 2048 outputs,
 * batch 1024, sigma 1, Adam lr 1e-3 (0.9, 0.999, 1e-8). */
void afd_mlp_default_params(afd_mlp_params* p);
int afd_mlp_create(afd_mlp** m, const afd_mlp_params* p);
void afd_mlp_destroy(afd_mlp* m);
const char* afd_mlp_last_error(const afd_mlp* m);  /* m = NULL: last create or GEMM failure */
int afd_mlp_set_stream(afd_mlp* m, void* stream);

/* One Adam step on n <= batch rows: x [n][n_in], y [n][n_out]. *loss (may
 * be NULL) receives the mean squared error before the step. */
int afd_mlp_train_step(afd_mlp* m, const float* x, const float* y, int32_t n, float* loss);
/* Gradients of the loss at the current weights, without an update. */
int afd_mlp_gradients(afd_mlp* m, const float* x, const float* y, int32_t n, float* loss);
/* out [n][n_out] = network(x). */
int afd_mlp_predict(afd_mlp* m, const float* x, int32_t n, float* out);
/* Waits for queued work; fails if a kernel wait expired. */
int afd_mlp_sync(afd_mlp* m);
int afd_mlp_get(afd_mlp* m, int32_t what, int32_t layer, float* out, int64_t cap);
int afd_mlp_set_weights(afd_mlp* m, int32_t layer, const float* w, const float* b);

/* C[M][N] (FP32, device) = A[M][K] * B[N][K]^T with A and B BF16 row-major
 * device arrays (K contiguous); M, N multiples of 128, K of 64. N a
 * multiple of 256 runs the persistent 128 x 256 tile kernel. Synchronises
 * the stream and fails if a kernel wait expired. */
int afd_gemm_bf16(const void* a, const void* b, float* c, int32_t M, int32_t N, int32_t K, void* stream);
/* The same GEMM queued on the stream without synchronising: a pipeline wait
 * that expired ORs 1 into *status (a device int32 the caller zeroes and
 * reads later). Usable inside stream capture. */
int afd_gemm_bf16_async(const void* a, const void* b, float* c, int32_t M, int32_t N, int32_t K, void* stream,
                        int32_t* status);

#ifdef __cplusplus
}
#endif

#endif
