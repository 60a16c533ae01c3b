/*
 * pdlpgpu_mlp.h -- the learned warm start: a 3-layer MLP (BF16 weights and
 * activations, FP32 accumulation) that maps an LP instance's parameters to a
 * starting point (x0, y0) and an initial primal weight, trained on the device
 * by this library's own tcgen05 tensor-core GEMM, backward and Adam kernels.
 *
 * No counterpart in the reference: its PdlpSolver::solve always starts from
 * the box projection of 0 and y = 0 with the option's primal weight
 * (pdlp_engine/src/pdlp_solver.cpp:168-176, pdlp_options.h:61-71). The solver
 * then runs from the prediction to the same tolerance; the better of the
 * prediction and the cold start by KKT score is used (pdlpgpu_warmstart).
 *
 * All tensors are device pointers, row-major:
 *   inputs   [batch][in]   BF16 (uint16 bit patterns)
 *   outputs  [batch][out]  FP32
 *   targets  [batch][out]  FP32, with per-output loss weights [out]
 * `in` must be a multiple of 8; `out` and `hidden` multiples of 64.
 * The model runs on its own stream, ordered after all work enqueued so far
 * on the legacy default stream (where the codec below and PyTorch enqueue
 * by default); arguments produced on another stream must be complete before
 * the call. Each call returns once its results are written.
 */
#ifndef PDLPGPU_MLP_H
#define PDLPGPU_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pdlpgpu_mlp pdlpgpu_mlp;

/* Weights He-initialised from `seed`; Adam state zero. Returns 0 or -1. */
int32_t pdlpgpu_mlp_create(int32_t in, int32_t hidden, int32_t out, int32_t batch,
                           uint64_t seed, int32_t device, pdlpgpu_mlp** mlp);
void pdlpgpu_mlp_destroy(pdlpgpu_mlp* mlp);

/* outputs = W3 relu(W2 relu(W1 x + b1) + b2) + b3 for `batch` rows. */
int32_t pdlpgpu_mlp_forward(pdlpgpu_mlp* mlp, const uint16_t* inputs, float* outputs);

/* One Adam step on the weighted mean-squared error
 * loss = (1/batch) sum_b sum_j w_j (out_bj - target_bj)^2.
 * Writes the loss (before the step) to *loss when non-NULL. */
int32_t pdlpgpu_mlp_train_step(pdlpgpu_mlp* mlp, const uint16_t* inputs, const float* targets,
                               const float* loss_weights, float learning_rate, float* loss);

/* Gradients of the loss at the current weights without updating them (for
 * gradient checks): device FP32 buffers shaped like the parameters, any may
 * be NULL. */
int32_t pdlpgpu_mlp_gradients(pdlpgpu_mlp* mlp, const uint16_t* inputs, const float* targets,
                              const float* loss_weights, float* dW1, float* db1, float* dW2,
                              float* db2, float* dW3, float* db3, float* loss);

/* Copies the FP32 master parameters out of / into the model (device
 * pointers, shapes W1 [hidden][in], b1 [hidden], W2 [hidden][hidden],
 * b2 [hidden], W3 [out][hidden], b3 [out]; NULL skips a tensor). Setting
 * refreshes the BF16 copies the GEMMs read. */
int32_t pdlpgpu_mlp_get_params(pdlpgpu_mlp* mlp, float* W1, float* b1, float* W2, float* b2,
                               float* W3, float* b3);
int32_t pdlpgpu_mlp_set_params(pdlpgpu_mlp* mlp, const float* W1, const float* b1,
                               const float* W2, const float* b2, const float* W3, const float* b3);

/* The tensor-core GEMM alone: C[M][N] (FP32) = A[M][K] * B[N][K]^T with A, B
 * BF16 row-major (K contiguous), K a multiple of 8, split over `splits`
 * K-ranges summed in a fixed order. Device pointers; returns 0 or -1. */
int32_t pdlpgpu_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* A, const uint16_t* B,
                          float* C, int32_t splits);

/* Measurement of the same GEMM (and, with splits > 1, the fixed-order sum of
 * the split-K partials): one warm-up call, then `reps` calls between CUDA
 * events on the legacy default stream; *ms_per_call is their mean. Scratch is
 * allocated before the first event. Returns 0 or -1. */
int32_t pdlpgpu_gemm_time(int32_t M, int32_t N, int32_t K, const uint16_t* A, const uint16_t* B,
                          float* C, int32_t splits, int32_t reps, double* ms_per_call);

/* Codec between an LP family's instances and the network (device pointers,
 * default stream). Features: the instance parameters [batch][count] (FP64)
 * standardised per feature and rounded to BF16, zero-padded to `padded`
 * columns. Targets: primal / primal_scale (the flow over its capacity), the
 * standardised row duals and the standardised log of the final primal
 * weight, zero-padded to out_width. Decoding inverts the targets and clamps
 * the primal to [0, primal_scale]; the result feeds pdlpgpu_session_load as
 * a warm start. Each returns 0 or -1. */
int32_t pdlpgpu_encode_features(const double* params, int32_t batch, int32_t count,
                                int32_t padded, const float* mean, const float* inv_std,
                                uint16_t* out);
int32_t pdlpgpu_encode_targets(const double* primal, const double* dual, const double* weight,
                               int32_t batch, int32_t n, int32_t m, int32_t out_width,
                               const double* primal_scale, const float* dual_mean,
                               const float* dual_inv_std, float weight_mean,
                               float weight_inv_std, float* targets);
int32_t pdlpgpu_decode_warmstart(const float* outputs, int32_t batch, int32_t n, int32_t m,
                                 int32_t out_width, const double* primal_scale,
                                 const float* dual_mean, const float* dual_std,
                                 float weight_mean, float weight_std, double* primal,
                                 double* dual, double* weight);

/* Kernel launches issued by the last forward / train step of `mlp`. */
int64_t pdlpgpu_mlp_launches(pdlpgpu_mlp* mlp);

#ifdef __cplusplus
}
#endif

#endif
