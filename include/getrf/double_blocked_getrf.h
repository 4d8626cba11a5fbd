/*
 * Double-blocked left-looking LU with partial pivoting, FP32.
 * Drop-in for reference include/getrf/double_blocked_getrf.h:9-60
 * (src/getrf/double_blocked_getrf.cpp:125-289,
 *  src/getrf/getrf_batched_pivot_internal.h:445-624).
 *
 * A (n x n, column-major, DEVICE) is overwritten by the packed unit-lower L
 * and upper U; ipiv (DEVICE, n ints) receives 1-based GLOBAL LAPACK pivots;
 * info (DEVICE int) is 0, the 1-based column of the first exact zero pivot, or
 * -1 for an invalid workspace / pivot (the reference's 0xff memset,
 * double_blocked_getrf.cpp:19-30).
 *
 * Pivot composition runs on the GPU: there is no host synchronisation per
 * panel (the reference copies pivots to the host and waits,
 * getrf_batched_pivot_internal.h:102-148).
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference double_blocked_getrf.h:9-19.  device_sources/device_targets hold
 * the composed row moves (capacity >= n ints each); device_swap_buffer backs
 * the two-pass row permutation when a permutation is too large for shared
 * memory (column_tile * capacity floats).  The host arrays are validated as in
 * the reference (getrf_batched_pivot_internal.h:43-57) but not used: pivots
 * are composed on the device. */
typedef struct getrf_batched_pivot_workspace {
    int* device_sources;
    int* device_targets;
    void* device_swap_buffer;
    int* host_pivots;
    int* host_permutation;
    int* host_sources;
    int* host_targets;
    int capacity;
    int column_tile;
} getrf_batched_pivot_workspace;

/* reference double_blocked_getrf.h:21-24 */
typedef enum getrf_outer_trsm_mode {
    getrf_outer_trsm_direct = 0,
    getrf_outer_trsm_iterative = 1
} getrf_outer_trsm_mode;

/* reference double_blocked_getrf.h:26-35: pivots applied immediately to every
 * column outside each panel. */
void double_blocked_getrf(hdbf_handle handle, float* A, int lda, int n, int outer_nb,
                          int inner_nb, getrf_outer_trsm_mode outer_trsm_mode,
                          int trsm_block, int* ipiv, int* info);

/* reference double_blocked_getrf.h:48-60: panel pivots applied inside the
 * current outer block only; the composed history permutation is applied to
 * the left block columns and to the next outer panel at each outer step. */
void double_blocked_getrf_batched_pivot(hdbf_handle handle, float* A, int lda, int n,
                                        int outer_nb, int inner_nb,
                                        getrf_outer_trsm_mode outer_trsm_mode,
                                        int trsm_block, int inner_gemm_m_tile, int* ipiv,
                                        int* info,
                                        getrf_batched_pivot_workspace* workspace);

/* reference double_blocked_getrf.h:37-46 (FP64 twin, immediate pivots) */
void double_blocked_getrf_double(hdbf_handle handle, double* A, int lda, int n, int outer_nb,
                                 int inner_nb, getrf_outer_trsm_mode outer_trsm_mode,
                                 int trsm_block, int* ipiv, int* info);

/* reference double_blocked_getrf.h:62-74 (FP64 twin, batched pivots); the
 * workspace's device_swap_buffer holds column_tile x n doubles. */
void double_blocked_getrf_double_batched_pivot(hdbf_handle handle, double* A, int lda, int n,
                                               int outer_nb, int inner_nb,
                                               getrf_outer_trsm_mode outer_trsm_mode,
                                               int trsm_block, int inner_gemm_m_tile, int* ipiv,
                                               int* info,
                                               getrf_batched_pivot_workspace* workspace);

#ifdef __cplusplus
}
#endif
