/*
 * Diagonal damping A <- A + lambda * I (n x n, column-major, DEVICE).
 * Drop-in for reference include/kernels/add_damping.h:12-27
 * (src/kernels/add_damping.hip:10-66).
 */
#pragma once
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

void launch_add_damping(float* A, int n, int lda, float lambda, cudaStream_t stream);
void launch_add_damping_double(double* A, int n, int lda, double lambda,
                               cudaStream_t stream);

#ifdef __cplusplus
}
#endif
