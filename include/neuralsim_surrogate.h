/*
 * neuralsim_surrogate.h — learned Hodgkin-Huxley macro-step (no counterpart
 * in the reference; it accelerates HodgkinHuxleyNeuron::step,
 * src/neuron/hodgkin_huxley.rs:46-96, as integrated by Rush-Larsen).
 *
 * The surrogate is an MLP 5 -> 128 -> 128 -> 4 with SiLU activations, BF16
 * weights and FP32 accumulation on the tensor cores (tcgen05). It maps the
 * state at the start of a 0.1 ms macro-step — membrane potential V, gates
 * m, h, n and the synaptic current I_syn held for the macro-step — to the
 * state 0.1 ms later, as 10 Rush-Larsen steps of 0.01 ms with that current
 * would produce it. Inputs and outputs are normalised: x' = (x - mean) /
 * scale for the inputs, and the outputs are the increments (V, m, h, n after
 * minus before) in the same form.
 *
 * Training runs on the GPU with this library's own forward and backward
 * kernels (BF16 tensor-core GEMMs, Adam in FP32). A handle owns the weights,
 * the optimizer state, a training set on the device and one CUDA stream.
 * Parameter order of the flat FP32 vector (17,796 values):
 *   W1 [128][5], b1 [128], W2 [128][128], b2 [128], W3 [4][128], b3 [4]
 * (row = output unit). Same conventions as neuralsim.h: ns_status returns,
 * host pointers are copied, no CPU fallback.
 */
#ifndef NEURALSIM_SURROGATE_H
#define NEURALSIM_SURROGATE_H

#include <stdint.h>

#include "neuralsim.h"

#ifdef __cplusplus
extern "C" {
#endif

#define NS_SUR_IN 5
#define NS_SUR_HIDDEN 128
#define NS_SUR_OUT 4
#define NS_SUR_PARAMS 17796
#define NS_SUR_SUBSTEPS 10

typedef struct ns_sur ns_sur;

/* HH parameters (g_na, g_k, g_l, e_na, e_k, e_l, c_m), the fine step (ms)
 * whose NS_SUR_SUBSTEPS Rush-Larsen steps make one macro-step, the training
 * batch (a multiple of 128) and the seed of the weight initialisation and
 * minibatch sampling. */
ns_status ns_sur_create(int device, const float hh_params[7], float dt_fine_ms, uint32_t batch,
                        uint64_t seed, ns_sur** out);
ns_status ns_sur_destroy(ns_sur* s);
const char* ns_sur_last_error(const ns_sur* s);

/* Training set: n states x[n][5] = (V, m, h, n, I_syn) (host). Targets are
 * computed on the device: NS_SUR_SUBSTEPS Rush-Larsen steps with I_syn held,
 * the arithmetic of the network step. y_out (host, [n][4], or NULL) receives
 * the states 0.1 ms later. */
ns_status ns_sur_set_data(ns_sur* s, const float* x, uint64_t n, float* y_out);

/* Normalisation: in_mean/in_scale [5] for the inputs, out_mean/out_scale [4]
 * for the increments. */
ns_status ns_sur_set_norm(ns_sur* s, const float in_mean[5], const float in_scale[5],
                          const float out_mean[4], const float out_scale[4]);

/* n_steps of Adam (beta 0.9 / 0.999, eps 1e-8) on minibatches drawn
 * uniformly (with replacement) from the training set; lr decays by
 * lr_decay per step. loss_out (host, n_steps or NULL): mean squared error of
 * the normalised increments of every step. */
ns_status ns_sur_train(ns_sur* s, uint32_t n_steps, float lr, float lr_decay, float* loss_out);

/* Data-parallel training, one process per GPU: ns_sur_grad_step draws one
 * minibatch from the training set and writes its loss gradient (flat order)
 * to grad_dev (device, NS_SUR_PARAMS floats) without an update; the caller
 * sums the gradients over ranks (one all-reduce of 17,796 floats) and
 * ns_sur_apply_gradient takes one Adam step with scale * grad_dev. Ranks
 * start from the same weights (ns_sur_set_params) and draw minibatches from
 * distinct streams (ns_sur_set_sample_seed). */
ns_status ns_sur_set_sample_seed(ns_sur* s, uint64_t seed);
ns_status ns_sur_grad_step(ns_sur* s, float* grad_dev, float* loss_out);
ns_status ns_sur_apply_gradient(ns_sur* s, const float* grad_dev, float scale, float lr);

/* Gradient of the minibatch loss at the current weights for the given batch
 * (host x[batch][5] raw states, y[batch][4] raw targets), without an update:
 * grad_out (host, NS_SUR_PARAMS) in the flat parameter order; loss_out (host
 * or NULL). For checking the backward kernels. */
ns_status ns_sur_gradient(ns_sur* s, const float* x, const float* y, float* grad_out,
                          float* loss_out);

/* Weights (host, NS_SUR_PARAMS floats, flat order). Setting them resets the
 * optimizer state. */
ns_status ns_sur_get_params(ns_sur* s, float* params);
ns_status ns_sur_set_params(ns_sur* s, const float* params);

/* Inference through the training kernels: x[n][5] raw -> y[n][4] raw states
 * 0.1 ms later (host arrays). */
ns_status ns_sur_predict(ns_sur* s, const float* x, uint64_t n, float* y);

/* BF16 tensor-core GEMM C[M][N] = A[M][K] * B[N][K]^T (device pointers,
 * row-major, K contiguous): M a multiple of 128, N 16 or 128, K a multiple
 * of 16, lda/ldb multiples of 8. epilogue 0: C = acc (+ bias[N]) fp32;
 * 1: C += acc (fp32 atomics) with K split over k_splits CTAs; 2: C = acc +
 * bias (fp32, C may be NULL) and H = bf16(silu(C)). stream: cudaStream_t. */
ns_status ns_tc_gemm_bf16(const uint16_t* A, const uint16_t* B, float* C, uint16_t* H,
                          const float* bias, uint32_t M, uint32_t N, uint32_t K, uint32_t lda,
                          uint32_t ldb, uint32_t ldc, uint32_t k_splits, int32_t epilogue,
                          void* stream);

/* Attaches a trained surrogate to a Hodgkin-Huxley handle (Rush-Larsen,
 * CONDUCTANCE_FRESH, windowed stepping with a window that is a multiple of
 * NS_SUR_SUBSTEPS, dt equal to the surrogate's fine step). Every later
 * macro-step of NS_SUR_SUBSTEPS steps advances a neuron with the MLP when
 * v_lo <= V <= v_hi at its start, the predicted V stays within [v_lo, v_hi]
 * and the trapezoidal residual of the predicted V is at most residual_mv;
 * otherwise with the plain Rush-Larsen steps. NULL detaches. */
ns_status ns_set_surrogate(ns_handle* h, const ns_sur* s, float v_lo, float v_hi,
                           float residual_mv);

/* What advances in-envelope neurons over a macro-step: 0 = the MLP (after
 * ns_set_surrogate); 1 = one Rush-Larsen step of the macro-step's length
 * (0.1 ms) with the same held current, envelope, residual check and fallback
 * — the plain method in the surrogate's cost class, for comparison; 2 = ten
 * Rush-Larsen steps of 0.01 ms with the held current — the function the MLP
 * is trained to reproduce, which separates the MLP's error from the error of
 * holding the synaptic current over a macro-step. */
ns_status ns_set_macro_step_mode(ns_handle* h, int32_t mode);

/* Neuron macro-steps taken by the surrogate and by the Rush-Larsen fallback
 * since the surrogate was attached. */
ns_status ns_surrogate_counts(ns_handle* h, uint64_t* by_mlp, uint64_t* by_fallback);

#ifdef __cplusplus
}
#endif
#endif /* NEURALSIM_SURROGATE_H */
