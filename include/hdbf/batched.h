/*
 * Batched uneven factor-and-solve in one persistent launch.  No counterpart in
 * the reference (which factors one matrix per call).
 *
 * count independent systems; system i has order n[i] (Cholesky <= 512, LU
 * <= 768), column-major DEVICE matrix A[i] (leading dimension lda[i]),
 * one DEVICE right-hand side b[i] (overwritten by the solution), and, for LU,
 * a DEVICE pivot array ipiv[i] (1-based, LAPACK order).  op[i] = 0 factors
 * with Cholesky (lower) and solves, op[i] = 1 with partially pivoted LU.
 * All pointer arrays (A, b, ipiv) and the integer arrays live in DEVICE
 * memory.  order[] is the processing order (e.g. by decreasing n^3 so the
 * longest systems start first); info[i] receives 0 or the 1-based first
 * failing column; queue is one DEVICE unsigned int the persistent CTAs use as
 * their work counter (reset by the call).
 *
 * variant selects the launch shape: threads per CTA (one matrix per CTA at a
 * time) and panel width, hdbf_batched_variant_shape; the panel width's
 * shared-memory footprint sets how many CTAs share an SM.  Variants 0, 1, 2
 * are 128, 256, 512 threads with 32-column panels; 3, 4, 5 the same with
 * 16-column panels.  The autotuner (hygondoubleblockedfactorizations_b200.tuner)
 * measures the variants on a batch and picks one.  The launch (queue reset +
 * kernel) is recorded once per argument tuple as a CUDA graph and replayed
 * afterwards.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

int hdbf_batched_num_variants(void);

/* Threads per CTA and panel width of a variant. */
hdbf_status hdbf_batched_variant_shape(int variant, int* threads, int* panel);

hdbf_status hdbf_batched_factor_solve(hdbf_handle handle, int variant, int count,
                                      const int* order, const int* op, const int* n,
                                      const int* lda, float* const* A, float* const* b,
                                      int* const* ipiv, int* info, unsigned int* queue);

#ifdef __cplusplus
}
#endif
