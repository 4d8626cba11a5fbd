/*
 * Classic blocked right-looking Cholesky (lower), FP32.
 * Drop-in for reference include/potrf/blocked_potrf.h:9-14
 * (src/potrf/blocked_potrf.cpp:126-206).
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void blocked_right_looking_potrf(hdbf_handle handle, float* A, int lda, int n, int nb,
                                 int* info);

/* reference blocked_potrf.h:16-20 (FP64 twin) */
void blocked_right_looking_potrf_double(hdbf_handle handle, double* A, int lda, int n, int nb,
                                        int* info);

#ifdef __cplusplus
}
#endif
