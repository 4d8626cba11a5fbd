/*
 * Double-blocked left-looking Cholesky (lower), FP32.
 * Drop-in for reference include/potrf/double_blocked_potrf.h:9-55
 * (implementation src/potrf/double_blocked_potrf.cpp:294-485).
 *
 * A is an n x n column-major DEVICE matrix (lda >= n); its lower triangle is
 * overwritten by L, the strict upper triangle is not modified.  nb is the outer
 * block, b the inner block (nb<=0 -> n, b<=0 -> nb, b=min(b,nb), as
 * double_blocked_potrf.cpp:309-321).  info is a DEVICE int: 0 on success,
 * else the 1-based global column of the first non-positive pivot (LAPACK
 * convention; the reference's block-local overwrite is not reproduced).
 * Every stage runs on this library's own sm_100a kernels.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference double_blocked_potrf.h:9-15 */
void double_blocked_potrf(hdbf_handle handle, float* A, int lda, int n, int nb, int b,
                          int* info);

/* reference double_blocked_potrf.h:17-23: panel TRSM run as a double-blocked
 * TRSM with micro-block 1024 (double_blocked_potrf.cpp:17, 79-119). */
void double_blocked_potrf_dbtrsm(hdbf_handle handle, float* A, int lda, int n, int nb,
                                 int b, int* info);

/* reference double_blocked_potrf.h:25-32: outer SYRK reduction split into
 * chunks of syrk_k_tile columns (src/syrk/kblocked_syrk.cpp:64-96). */
void double_blocked_potrf_kblocked_syrk(hdbf_handle handle, float* A, int lda, int n,
                                        int nb, int b, int syrk_k_tile, int* info);

/* reference double_blocked_potrf.h:34-42: as above plus inner-GEMM M-tiling
 * (tile 8192 when rows > 32768 and k >= 5632, double_blocked_potrf.cpp:17-20). */
void double_blocked_potrf_kblocked_syrk_adaptive_gemm(hdbf_handle handle, float* A,
                                                      int lda, int n, int nb, int b,
                                                      int syrk_k_tile, int* info);

/* reference double_blocked_potrf.h:44-55 */
void double_blocked_potrf_kblocked_syrk_adaptive_gemm_configured(
    hdbf_handle handle, float* A, int lda, int n, int nb, int b, int syrk_k_tile,
    int gemm_m_tile, int gemm_m_threshold, int gemm_k_threshold, int* info);

/* FP64 twins (reference double_blocked_potrf.h:57-103): same arguments and
 * info convention, double-precision storage and arithmetic throughout. */
/* reference double_blocked_potrf.h:57-63 */
void double_blocked_potrf_double(hdbf_handle handle, double* A, int lda, int n, int nb, int b,
                                 int* info);
/* reference double_blocked_potrf.h:65-71 */
void double_blocked_potrf_double_dbtrsm(hdbf_handle handle, double* A, int lda, int n, int nb,
                                        int b, int* info);
/* reference double_blocked_potrf.h:73-80 */
void double_blocked_potrf_double_kblocked_syrk(hdbf_handle handle, double* A, int lda, int n,
                                               int nb, int b, int syrk_k_tile, int* info);
/* reference double_blocked_potrf.h:82-90 */
void double_blocked_potrf_double_kblocked_syrk_adaptive_gemm(hdbf_handle handle, double* A,
                                                             int lda, int n, int nb, int b,
                                                             int syrk_k_tile, int* info);
/* reference double_blocked_potrf.h:92-103 */
void double_blocked_potrf_double_kblocked_syrk_adaptive_gemm_configured(
    hdbf_handle handle, double* A, int lda, int n, int nb, int b, int syrk_k_tile,
    int gemm_m_tile, int gemm_m_threshold, int gemm_k_threshold, int* info);

#ifdef __cplusplus
}
#endif
