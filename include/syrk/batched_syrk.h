/*
 * Bottom-up batched lower SYRK C_lower -= A * A^T.
 * Drop-in for reference include/syrk/batched_syrk.h:24-43
 * (src/syrk/batched_syrk.cpp:27-153, 284-407): nb x nb diagonal leaves plus
 * off-diagonal GEMM merges.  The FP32 variant runs the SIMT FP32 kernels; the
 * _mixed variant runs tcgen05 FP16 tiles with FP32 accumulation and FP32 C.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void batched_syrk_bottom_up(hdbf_handle handle, StreamPool* pool, float* A, int lda,
                            float* C, int ldc, int n, int k, int nb);


/* reference batched_syrk.h:40-43: FP16 tensor-core products, FP32 C. */
void batched_syrk_bottom_up_mixed(hdbf_handle handle, StreamPool* pool, float* A, int lda,
                                  float* C, int ldc, int n, int k, int nb);

/* reference batched_syrk.h:32-35 (FP64 twin; the pool is accepted, the work
 * runs on the handle's stream) */
void batched_syrk_bottom_up_double(hdbf_handle handle, StreamPool* pool, double* A, int lda,
                                   double* C, int ldc, int n, int k, int nb);

#ifdef __cplusplus
}
#endif
