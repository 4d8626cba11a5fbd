/*
 * Double-blocked right/lower/transposed TRSM, FP32.
 * Drop-in for reference include/trsm/double_blocked_trsm.h:9-17
 * (src/trsm/double_blocked_trsm.cpp:99-171): B (n x m) <- B * A^{-T},
 * A lower m x m, outer block nb and inner block b.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void double_blocked_trsm(hdbf_handle handle, float* A, int lda, float* B, int ldb, int n,
                         int m, int nb, int b);

/* reference double_blocked_trsm.h:19-27 (FP64 twin) */
void double_blocked_trsm_double(hdbf_handle handle, double* A, int lda, double* B, int ldb,
                                int n, int m, int nb, int b);

#ifdef __cplusplus
}
#endif
