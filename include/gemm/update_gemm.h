/*
 * Trailing update C -= A * B^T, FP32 (SIMT FFMA tiles).
 * Drop-in for reference include/gemm/update_gemm.h:9-41
 * (src/gemm/update_gemm.cpp:10-101).  C is rows x cols, A rows x k, B cols x k.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference update_gemm.h:9-18 */
void gemm_nt_update(hdbf_handle handle, int rows, int cols, int k, const float* A, int lda,
                    const float* B, int ldb, float* C, int ldc);

/* reference update_gemm.h:31-41: rows processed in m_tile chunks (m_tile <= 0:
 * one pass) */
void gemm_nt_update_m_tiled(hdbf_handle handle, int rows, int cols, int k, const float* A,
                            int lda, const float* B, int ldb, float* C, int ldc,
                            int m_tile);

/* reference update_gemm.h:20-29 (FP64 twin): C -= A * B^T */
void gemm_nt_update_double(hdbf_handle handle, int rows, int cols, int k, const double* A,
                           int lda, const double* B, int ldb, double* C, int ldc);

/* reference update_gemm.h:43-52 (FP64 twin) */
void gemm_nt_update_m_tiled_double(hdbf_handle handle, int rows, int cols, int k,
                                   const double* A, int lda, const double* B, int ldb,
                                   double* C, int ldc, int m_tile);

#ifdef __cplusplus
}
#endif
