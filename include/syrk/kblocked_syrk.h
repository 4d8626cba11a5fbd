/*
 * Lower SYRK trailing update C_lower -= A * A^T, FP32.
 * Drop-in for reference include/syrk/kblocked_syrk.h:9-41
 * (src/syrk/kblocked_syrk.cpp:18-96).  C is n x n, A is n x k; only the lower
 * triangle of C (diagonal included) is read or written.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference kblocked_syrk.h:9-15 */
void syrk_lower_update(hdbf_handle handle, int n, int k, const float* A, int lda, float* C,
                       int ldc);

/* reference kblocked_syrk.h:25-32: reduction split into k_tile chunks
 * (k_tile <= 0 or >= k: one pass). */
void syrk_lower_update_kblocked(hdbf_handle handle, int n, int k, const float* A, int lda,
                                float* C, int ldc, int k_tile);

/* reference kblocked_syrk.h:17-23 (FP64 twin) */
void syrk_lower_update_double(hdbf_handle handle, int n, int k, const double* A, int lda,
                              double* C, int ldc);

/* reference kblocked_syrk.h:34-41 (FP64 twin) */
void syrk_lower_update_kblocked_double(hdbf_handle handle, int n, int k, const double* A,
                                       int lda, double* C, int ldc, int k_tile);

#ifdef __cplusplus
}
#endif
