/*
 * Row-interchange kernels, FP32.
 * Drop-in for reference include/getrf/getrf_pivot_kernels.h:9-43
 * (src/getrf/getrf_pivot_kernels.hip:14-206).
 */
#pragma once
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

/* reference getrf_pivot_kernels.h:9-15: apply the panel's LAPACK-order swaps
 * (pivots are 1-based rows local to A(panel:n, :)) to every column outside
 * [panel, panel+panel_size), then globalise pivots in place (+panel).  The
 * swaps are composed into one row permutation on the GPU and applied with a
 * column-tiled gather/scatter (the reference swaps sequentially, one thread
 * per column).  Uses a small internal device buffer created on first use. */
void launch_apply_getrf_panel_pivots(float* A, int lda, int n, int panel, int panel_size,
                                     int* pivots, cudaStream_t stream);

/* reference getrf_pivot_kernels.h:25-33: A[targets[m], c] = old A[sources[m], c]
 * for every column c < column_count, staged through `temporary`
 * (column_tile * move_count floats) one column tile at a time. */
void launch_apply_getrf_permutation(float* A, int lda, int column_count,
                                    const int* sources, const int* targets, int move_count,
                                    float* temporary, int column_tile,
                                    cudaStream_t stream);

/* reference getrf_pivot_kernels.h:17-23 (FP64 twin) */
void launch_apply_getrf_panel_pivots_double(double* A, int lda, int n, int panel,
                                            int panel_size, int* pivots, cudaStream_t stream);

/* reference getrf_pivot_kernels.h:35-43 (FP64 twin); temporary holds
 * column_tile x move_count doubles. */
void launch_apply_getrf_permutation_double(double* A, int lda, int column_count,
                                           const int* sources, const int* targets,
                                           int move_count, double* temporary, int column_tile,
                                           cudaStream_t stream);

#ifdef __cplusplus
}
#endif
