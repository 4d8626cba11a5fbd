/*
 * Recursive Cholesky (lower), FP32.
 * Drop-in for reference include/potrf/recursive_potrf.h:10-37
 * (src/potrf/recursive_potrf.cpp:17-174, 241-388).
 *
 * Splits n -> n/2 until n <= nb, then factors the leaf with this library's
 * blocked diagonal kernel.  `pool` may be NULL; all work is stream-ordered on
 * the handle's stream (the reference's per-level host synchronisation of pool
 * streams, src/syrk/batched_syrk.cpp:15-22, is not needed).
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference recursive_potrf.h:10-15 */
void recursive_potrf(hdbf_handle handle, StreamPool* pool, float* A, int lda, int n,
                     int nb, int* info);

/* reference recursive_potrf.h:17-22 (TRSM updates tiled at 8192,
 * src/trsm/recursive_trsm.cpp:12, 82-122) */
void recursive_potrf_tiled_trsm(hdbf_handle handle, StreamPool* pool, float* A, int lda,
                                int n, int nb, int* info);


/* reference recursive_potrf.h:31-37.  Mixed-precision Cholesky: FP32 panels
 * and FP16 tensor-core (tcgen05) trailing updates with FP32 accumulation and
 * FP32 C (the reference rounds C to FP16, mixed_gemm.cpp:53-89), block nb.
 * On a failed factorization it keeps the reference's damping retry: restore A,
 * add lambda*I (lambda0 = 1e-4 * max|a_ii|, the reference's 6.55 on its
 * 65504-scaled matrix), double lambda, at most 5 attempts
 * (recursive_potrf.cpp:288-314, 375).  Synchronises the stream. */
void recursive_potrf_mixed_driver(hdbf_handle handle, StreamPool* pool, float* A, int lda,
                                  int n, int nb, int* info);

/* reference recursive_potrf.h:24-29 (FP64 twin; the pool is accepted and,
 * as in the FP32 entry point, the work runs on the handle's stream) */
void recursive_potrf_double(hdbf_handle handle, StreamPool* pool, double* A, int lda, int n,
                            int nb, int* info);

#ifdef __cplusplus
}
#endif
