/*
 * Blocked right-looking LU without pivoting, FP32.
 * Drop-in for reference include/getrf/blocked_getrf_npvt.h:9-14
 * (src/getrf/blocked_getrf_npvt.cpp).
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void blocked_right_looking_getrf_npvt(hdbf_handle handle, float* A, int lda, int n,
                                      int nb, int* info);

/* reference blocked_getrf_npvt.h:16-20 (FP64 twin) */
void blocked_right_looking_getrf_npvt_double(hdbf_handle handle, double* A, int lda, int n,
                                             int nb, int* info);

#ifdef __cplusplus
}
#endif
