/*
 * Recursive lower SYRK C_lower -= A * A^T, FP32.
 * Drop-in for reference include/syrk/recursive_syrk.h:15-20
 * (src/syrk/recursive_syrk.cpp:9-89): diagonal halves recursively, the
 * off-diagonal block as one GEMM; stream-ordered on the handle's stream.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void recursive_syrk_parallel(hdbf_handle handle, float* A, int lda, float* C, int ldc,
                             int n, int k, int nb);

/* reference recursive_syrk.h:25-30 (FP64 twin) */
void recursive_syrk_parallel_double(hdbf_handle handle, double* A, int lda, double* C, int ldc,
                                    int n, int k, int nb);

#ifdef __cplusplus
}
#endif
