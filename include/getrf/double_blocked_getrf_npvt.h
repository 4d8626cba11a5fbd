/*
 * Double-blocked left-looking LU without pivoting, FP32.
 * Drop-in for reference include/getrf/double_blocked_getrf_npvt.h:9-15
 * (src/getrf/double_blocked_getrf_npvt.cpp:93-144).
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void double_blocked_getrf_npvt(hdbf_handle handle, float* A, int lda, int n, int nb,
                               int b, int* info);

/* reference double_blocked_getrf_npvt.h:17-23 (FP64 twin) */
void double_blocked_getrf_npvt_double(hdbf_handle handle, double* A, int lda, int n, int nb,
                                      int b, int* info);

#ifdef __cplusplus
}
#endif
