/*
 * CPU restatement of the reference's double-blocked factorization loops --
 * TEST INFRASTRUCTURE ONLY (never linked into, or called by, the CUDA library).
 *
 * Plain loops (FP32, and FP64 for the `_double` twins) that follow the
 * reference schedules step for step, with the
 * vendor library calls (rocsolver_spotrf / rocsolver_sgetrf / rocblas_strsm /
 * rocblas_sgemm / rocblas_ssyrk) replaced by their textbook LAPACK/BLAS
 * definitions:
 *
 *   oracle_double_blocked_potrf  src/potrf/double_blocked_potrf.cpp:294-381
 *       update_next_inner_panel  src/potrf/double_blocked_potrf.cpp:210-249
 *       prepare_next_outer_panel src/potrf/double_blocked_potrf.cpp:251-292
 *   oracle_double_blocked_getrf  src/getrf/double_blocked_getrf.cpp:125-191
 *   oracle_double_blocked_getrf_batched
 *                                src/getrf/getrf_batched_pivot_internal.h:445-624
 *   oracle_recursive_potrf       src/potrf/recursive_potrf.cpp:17-174
 *   oracle_blocked_right_looking_potrf  src/potrf/blocked_potrf.cpp:127-181
 *   oracle_blocked_right_looking_getrf  src/getrf/blocked_getrf.cpp:15-71
 *                                       (pivot = 0: blocked_getrf_npvt.cpp)
 *       prepare_next_inner_panel src/getrf/double_blocked_getrf.cpp:32-71
 *       prepare_next_outer_panel src/getrf/double_blocked_getrf.cpp:73-123
 *       apply_panel_pivots       src/getrf/getrf_pivot_kernels.hip:14-45
 *
 * The unblocked kernels follow LAPACK's reference definitions:
 *   potf2: left-looking, a_jj -= dot, sqrt, column scaled by 1/a_jj (xPOTF2)
 *   getf2: ISAMAX (first maximum), row swap, scale by 1/pivot when
 *          |pivot| >= sfmin else divide, rank-1 update (xGETF2)
 * info follows LAPACK: first global failing column, 1-based (the reference's
 * per-call overwrite of info is a documented quirk not reproduced).
 */
#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#define AT(A, lda, i, j) ((A)[(size_t)(j) * (size_t)(lda) + (size_t)(i)])

static int imin(int a, int b) { return a < b ? a : b; }

/* FP32: the reference's float entry points. */
#define REAL float
#define F(name) name##_f32
#define SQRT sqrtf
#define FABS fabsf
#define SFMIN FLT_MIN
#include "factor_impl.h"
#undef REAL
#undef F
#undef SQRT
#undef FABS
#undef SFMIN

/* FP64: the reference's `_double` entry points
 * (include/potrf/double_blocked_potrf.h:57-103,
 * include/getrf/double_blocked_getrf.h:37-46), same loops in double. */
#define REAL double
#define F(name) name##_f64
#define SQRT sqrt
#define FABS fabs
#define SFMIN DBL_MIN
#include "factor_impl.h"
#undef REAL
#undef F
#undef SQRT
#undef FABS
#undef SFMIN

int oracle_double_blocked_potrf(float* A, int lda, int n, int nb, int b, int syrk_k_tile)
{
    return oracle_double_blocked_potrf_f32(A, lda, n, nb, b, syrk_k_tile);
}

int oracle_double_blocked_getrf(float* A, int lda, int n, int outer_nb, int inner_nb, int* ipiv)
{
    return oracle_double_blocked_getrf_f32(A, lda, n, outer_nb, inner_nb, ipiv);
}
