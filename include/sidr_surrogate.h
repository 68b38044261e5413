/*
 * sidr_surrogate.h -- C-ABI of the surrogate-assisted GP (no counterpart in
 * the reference, which evaluates every offspring in full).
 *
 * A rule's phenotype -- its priority ranking on fixed decision situations
 * recorded from simulator rollouts, plus token-count features -- feeds a
 * 40 -> 256 -> 256 -> 1 ReLU MLP with BF16 weights and activations and FP32
 * accumulation whose GEMMs run on hand-written sm_100a tensor-core kernels
 * (tcgen05.mma with TMEM accumulators).  The model is trained online on the
 * fitness the simulator has just produced and pre-screens GP offspring; the
 * simulator stays the judge of every reported fitness, and the GP falls back
 * to plain breeding when the model's rank correlation on an audit sample is
 * too low.
 */
#ifndef SIDR_SURROGATE_H
#define SIDR_SURROGATE_H

#include <stdint.h>

#include "sidr.h"
#include "sidr_gp.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SIDR_MLP_INPUTS 40
#define SIDR_MLP_HIDDEN 256

/* C[M x N] (FP32) = A[M x K] * B[N x K]^T with BF16 operands given as raw
 * 16-bit patterns, on the tensor-core kernel the model uses (diagnostic).
 * splits > 1 splits K over CTAs that accumulate atomically.  N <= 256. */
sidr_status sidr_gemm_bf16(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K,
                           int32_t splits, int device, float* C);

/* The model: parameters 0 W1 [256 x 48] (input columns 40..47 are zero
 * padding), 1 b1 [256], 2 W2 [256 x 256], 3 b2 [256], 4 w3 [256], 5 b3 [1],
 * FP32 masters with BF16 copies for the GEMMs; He-uniform initialisation
 * from seed. */
typedef struct sidr_mlp sidr_mlp;
sidr_status sidr_mlp_create(int device, uint64_t seed, sidr_mlp** out);
void sidr_mlp_destroy(sidr_mlp* m);

/* Reads (write = 0) or replaces (write = 1) parameter `which`'s FP32 values;
 * grads (may be NULL) receives its gradient from the last sidr_mlp_gradients
 * or training step; *count its size. */
sidr_status sidr_mlp_param(sidr_mlp* m, int32_t which, int32_t write, float* values, float* grads,
                           int64_t* count);

/* y[rows] = model(x[rows][40]). */
sidr_status sidr_mlp_predict(sidr_mlp* m, const float* x, int32_t rows, float* y);

/* Mean squared error of the model on (x, t) and the gradients of every
 * parameter (read them with sidr_mlp_param); no update. */
sidr_status sidr_mlp_gradients(sidr_mlp* m, const float* x, const float* t, int32_t rows, float* loss);

/* `steps` Adam steps (beta 0.9 / 0.999, eps 1e-8) of `batch` rows drawn
 * without replacement from (x[n][40], t[n]), reshuffled every pass. */
sidr_status sidr_mlp_train(sidr_mlp* m, const float* x, const float* t, int32_t n, int32_t steps,
                           int32_t batch, float lr, uint64_t seed, float* final_loss);

#ifdef __cplusplus
}
#endif
#endif
