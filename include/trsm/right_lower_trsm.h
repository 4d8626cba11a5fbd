/*
 * Right, lower, transposed, non-unit triangular solve B <- B * L^{-T}, FP32.
 * Drop-in for reference include/trsm/right_lower_trsm.h:9-15
 * (src/trsm/right_lower_trsm.cpp:9-55).  B is rows x cols, L is cols x cols.
 */
#pragma once
#include <cuda_runtime_api.h>
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void trsm_right_lower_transpose(hdbf_handle handle, int rows, int cols, const float* A,
                                int lda, float* B, int ldb);

/* Largest `cols` accepted by trsm_right_lower_transpose_noalloc. */
#define HDBF_NOALLOC_TRSM_MAX_COLS 4096

/* No counterpart in the reference.  Same solve as trsm_right_lower_transpose
 * for callers that must not allocate device memory (services whose device
 * memory is fixed at start-up, libraries that may only use caller-owned
 * buffers): it takes a bare stream
 * instead of a handle and performs no cudaMalloc / cudaFree.  Its only
 * scratch, the inverted 64x64 diagonal blocks of A, lives in a 1 MiB device
 * array inside the library that every GPU loading the library keeps until the
 * process exits.  cols > HDBF_NOALLOC_TRSM_MAX_COLS returns
 * HDBF_STATUS_INVALID_VALUE and leaves B untouched.  The first call on a
 * device looks up that array's device address (cudaGetSymbolAddress) with the
 * device current.  All calls share the one array and leave their last contents in
 * it; calls that overlap on the GPU (different streams, or different host
 * threads without ordering) race on it. */
hdbf_status trsm_right_lower_transpose_noalloc(int rows, int cols, const float* A, int lda,
                                               float* B, int ldb, cudaStream_t stream);

/* reference right_lower_trsm.h:17-23 (FP64 twin): B <- B * L^{-T} */
void trsm_right_lower_transpose_double(hdbf_handle handle, int rows, int cols, const double* A,
                                       int lda, double* B, int ldb);

#ifdef __cplusplus
}
#endif
