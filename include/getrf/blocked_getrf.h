/*
 * Blocked right-looking LU with partial pivoting, FP32.
 * Drop-in for reference include/getrf/blocked_getrf.h:9-15
 * (src/getrf/blocked_getrf.cpp:15-71).
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void blocked_right_looking_getrf(hdbf_handle handle, float* A, int lda, int n, int nb,
                                 int* ipiv, int* info);

/* reference blocked_getrf.h:17-22 (FP64 twin) */
void blocked_right_looking_getrf_double(hdbf_handle handle, double* A, int lda, int n, int nb,
                                        int* ipiv, int* info);

#ifdef __cplusplus
}
#endif
