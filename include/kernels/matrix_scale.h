/*
 * SPD auto-scaling: forward scales the lower triangle by 65504 / max|diag|,
 * inverse multiplies the factor's lower triangle by sqrt(max / 65504).
 * Drop-in for reference include/kernels/matrix_scale.h:4-26
 * (src/kernels/matrix_scale.hip:10-113).  d_max_val (DEVICE) keeps the
 * maximum as FP32 bits between the forward and the inverse call.
 */
#pragma once
#include <stdbool.h>
#include <cuda_runtime_api.h>

#define HDBF_SCALE_TARGET 65504.0f

#ifdef __cplusplus
extern "C" {
#endif

void launch_auto_scale(float* A, int n, int lda, unsigned int* d_max_val, bool inverse,
                       cudaStream_t stream);

#ifdef __cplusplus
}
#endif
