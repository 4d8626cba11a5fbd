/*
 * Learned configuration selector (3-layer FP32 MLP, 64 hidden units) with its
 * own GPU kernels.  No counterpart in the reference, which picks the outer
 * and inner blocks by fixed policies (src/potrf/double_blocked_potrf.cpp:17-20,
 * 232-233; src/getrf/double_blocked_getrf.cpp:137-146 clamps nb/b) and sweeps
 * them by hand in its benchmark cases
 * (src/potrf/benchmark/potrf_double_blocked_cases.cpp:11-114,
 * src/getrf/benchmark/getrf_double_blocked_cases.cpp:12-109).
 *
 * Network: x (F features) -> relu(x W1 + b1) -> relu(. W2 + b2) -> z = . W3 + b3
 * (K candidate scores).  Parameters are one flat FP32 DEVICE array in the
 * order W1 (F x 64, row-major), b1 (64), W2 (64 x 64), b2 (64), W3 (64 x K),
 * b3 (K).  Samples are row-major DEVICE arrays: X (N x F), soft targets
 * Q (N x K, rows summing to 1 over the valid candidates) and mask (N x K,
 * 1 = the candidate applies to the sample, 0 = it does not).
 */
#pragma once
#include "hdbf/hdbf.h"

#define HDBF_SELECTOR_HIDDEN 64
#define HDBF_SELECTOR_MAX_FEATURES 32
#define HDBF_SELECTOR_MAX_CLASSES 32

#ifdef __cplusplus
extern "C" {
#endif

/* Number of parameters for F features and K classes (-1 if out of range). */
int hdbf_selector_num_params(int num_features, int num_classes);

/* Glorot-uniform weights from the library's counter-based U[-1,1) stream
 * (seeded), zero biases. */
hdbf_status hdbf_selector_init(hdbf_handle handle, float* theta, int num_features,
                               int num_classes, unsigned long long seed);

/* Full-batch Adam (beta1 0.9, beta2 0.999, eps 1e-8, L2 weight decay added to
 * the gradient) on the mean masked-softmax cross-entropy, `epochs` steps in
 * one launch.  step0 = Adam steps already taken (bias correction); adam_m and
 * adam_v (num_params floats each, zero before the first call) carry the
 * moments between calls.  loss_out (optional, `epochs` floats) receives the
 * loss before each step.  epochs == 0 evaluates only: loss_out[0] and, if
 * grad_out is given, the gradient at theta (no update, no weight decay). */
hdbf_status hdbf_selector_train(hdbf_handle handle, float* theta, float* adam_m, float* adam_v,
                                int step0, const float* X, const float* Q, const float* mask,
                                int num_samples, int num_features, int num_classes, int epochs,
                                float lr, float weight_decay, float* loss_out, float* grad_out);

/* Per sample: cls = argmax over valid candidates, conf = its softmax
 * probability, probs (optional, N x K) = the masked softmax. */
hdbf_status hdbf_selector_predict(hdbf_handle handle, const float* theta, const float* X,
                                  const float* mask, int num_samples, int num_features,
                                  int num_classes, int* cls, float* conf, float* probs);

#ifdef __cplusplus
}
#endif
