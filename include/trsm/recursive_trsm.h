/*
 * Recursive right/lower/transposed TRSM B (n x m) <- B * A^{-T}, FP32.
 * Drop-in for reference include/trsm/recursive_trsm.h:13-45
 * (src/trsm/recursive_trsm.cpp:132-378).
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference recursive_trsm.h:13-17: split m in halves down to nb */
void recursive_trsm(hdbf_handle handle, float* A, int lda, float* B, int ldb, int n, int m,
                    int nb);

/* reference recursive_trsm.h:19-23: update GEMMs tiled at 8192 */
void recursive_trsm_tiled_update(hdbf_handle handle, float* A, int lda, float* B, int ldb,
                                 int n, int m, int nb);


/* reference recursive_trsm.h:35-45: update GEMMs on FP16 tensor cores with
 * FP32 accumulation and FP32 B; FP32 leaves of order <= nb. */
void recursive_trsm_mixed(hdbf_handle handle, float* A, int lda, float* B, int ldb, int n, int m,
                          int nb);

/* reference recursive_trsm.h:29-33 (FP64 twin) */
void recursive_trsm_double(hdbf_handle handle, double* A, int lda, double* B, int ldb, int n,
                           int m, int nb);

#ifdef __cplusplus
}
#endif
