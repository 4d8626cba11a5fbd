/*
 * CPU restatement of the reference's double-blocked factorization loops --
 * TEST INFRASTRUCTURE ONLY (never linked into, or called by, the CUDA library).
 *
 * Plain FP32 loops that follow the reference schedules step for step, with the
 * vendor library calls (rocsolver_spotrf / rocsolver_sgetrf / rocblas_strsm /
 * rocblas_sgemm / rocblas_ssyrk) replaced by their textbook LAPACK/BLAS
 * definitions:
 *
 *   oracle_double_blocked_potrf  src/potrf/double_blocked_potrf.cpp:294-381
 *       update_next_inner_panel  src/potrf/double_blocked_potrf.cpp:210-249
 *       prepare_next_outer_panel src/potrf/double_blocked_potrf.cpp:251-292
 *   oracle_double_blocked_getrf  src/getrf/double_blocked_getrf.cpp:125-191
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

/* LAPACK xPOTF2 (lower): returns 0 or the 1-based local failing column. */
static int potf2_lower(int n, float* A, int lda)
{
    for (int j = 0; j < n; ++j) {
        float ajj = AT(A, lda, j, j);
        for (int k = 0; k < j; ++k) ajj -= AT(A, lda, j, k) * AT(A, lda, j, k);
        if (!(ajj > 0.0f)) {
            AT(A, lda, j, j) = ajj;
            return j + 1;
        }
        ajj = sqrtf(ajj);
        AT(A, lda, j, j) = ajj;
        for (int i = j + 1; i < n; ++i) {
            float s = AT(A, lda, i, j);
            for (int k = 0; k < j; ++k) s -= AT(A, lda, i, k) * AT(A, lda, j, k);
            AT(A, lda, i, j) = s;
        }
        float r = 1.0f / ajj;
        for (int i = j + 1; i < n; ++i) AT(A, lda, i, j) *= r;
    }
    return 0;
}

/* B (rows x cols) <- B * L^{-T}, L lower non-unit cols x cols. */
static void trsm_right_lower_trans(int rows, int cols, const float* L, int ldl,
                                   float* B, int ldb)
{
    for (int i = 0; i < rows; ++i) {
        for (int j = 0; j < cols; ++j) {
            float s = AT(B, ldb, i, j);
            for (int k = 0; k < j; ++k) s -= AT(B, ldb, i, k) * AT(L, ldl, j, k);
            AT(B, ldb, i, j) = s / AT(L, ldl, j, j);
        }
    }
}

/* C (rows x cols) -= A (rows x k) * B^T, B is cols x k. */
static void gemm_nt_sub(int rows, int cols, int k, const float* A, int lda,
                        const float* B, int ldb, float* C, int ldc)
{
    for (int j = 0; j < cols; ++j)
        for (int p = 0; p < k; ++p) {
            float b = AT(B, ldb, j, p);
            for (int i = 0; i < rows; ++i) AT(C, ldc, i, j) -= AT(A, lda, i, p) * b;
        }
}

/* C_lower (n x n) -= A (n x k) * A^T. */
static void syrk_lower_sub(int n, int k, const float* A, int lda, float* C, int ldc)
{
    for (int j = 0; j < n; ++j)
        for (int p = 0; p < k; ++p) {
            float b = AT(A, lda, j, p);
            for (int i = j; i < n; ++i) AT(C, ldc, i, j) -= AT(A, lda, i, p) * b;
        }
}

/* C (rows x cols) -= L (rows x k) * U (k x cols). */
static void gemm_nn_sub(int rows, int cols, int k, const float* L, int ldl,
                        const float* U, int ldu, float* C, int ldc)
{
    for (int j = 0; j < cols; ++j)
        for (int p = 0; p < k; ++p) {
            float u = AT(U, ldu, p, j);
            for (int i = 0; i < rows; ++i) AT(C, ldc, i, j) -= AT(L, ldl, i, p) * u;
        }
}

/* B (rows x cols) <- L^{-1} B, L unit lower rows x rows. */
static void trsm_left_lower_unit(int rows, int cols, const float* L, int ldl,
                                 float* B, int ldb)
{
    for (int j = 0; j < cols; ++j)
        for (int p = 0; p < rows; ++p) {
            float x = AT(B, ldb, p, j);
            for (int i = p + 1; i < rows; ++i) AT(B, ldb, i, j) -= AT(L, ldl, i, p) * x;
        }
}

/*
 * Double-blocked left-looking Cholesky, lower
 * (src/potrf/double_blocked_potrf.cpp:294-381).  nb<=0 -> n, b<=0 -> nb,
 * b = min(b, nb) (:309-321).  syrk_k_tile > 0 splits the outer SYRK's
 * reduction into chunks (src/syrk/kblocked_syrk.cpp:64-96).
 */
int oracle_double_blocked_potrf(float* A, int lda, int n, int nb, int b,
                                int syrk_k_tile)
{
    int info = 0;
    if (n <= 0) return 0;
    if (nb <= 0) nb = n;
    if (b <= 0) b = nb;
    b = imin(b, nb);
    for (int outer = 0; outer < n; outer += nb) {
        int outer_end = outer + imin(nb, n - outer);
        for (int inner = outer; inner < outer_end; inner += b) {
            int isz = imin(b, outer_end - inner);
            int ps = inner + isz;
            int f = potf2_lower(isz, &AT(A, lda, inner, inner), lda);
            if (f && !info) info = inner + f;
            trsm_right_lower_trans(n - ps, isz, &AT(A, lda, inner, inner), lda,
                                   &AT(A, lda, ps, inner), lda);
            if (ps < outer_end) {
                int pc = imin(b, outer_end - ps);
                /* full rectangle (rows ps..n) x (cols ps..ps+pc); the
                 * reference's GEMM also rewrites the diagonal block's strict
                 * upper triangle, which is never read back. */
                gemm_nt_sub(n - ps, pc, ps - outer, &AT(A, lda, ps, outer), lda,
                            &AT(A, lda, ps, outer), lda, &AT(A, lda, ps, ps), lda);
            }
        }
        if (outer_end < n) {
            int next = outer_end;
            int nsz = imin(nb, n - next);
            int below = next + nsz;
            int tk = syrk_k_tile > 0 ? syrk_k_tile : next;
            for (int k0 = 0; k0 < next; k0 += tk) {
                int kc = imin(tk, next - k0);
                syrk_lower_sub(nsz, kc, &AT(A, lda, next, k0), lda,
                               &AT(A, lda, next, next), lda);
            }
            gemm_nt_sub(n - below, nsz, next, &AT(A, lda, below, 0), lda,
                        &AT(A, lda, next, 0), lda, &AT(A, lda, below, next), lda);
        }
    }
    return info;
}

/*
 * LAPACK xGETF2 on an m x w panel: local 1-based pivots into ipiv[0..w),
 * returns 0 or the 1-based local column of the first exact zero pivot.
 */
static int getf2(int m, int w, float* A, int lda, int* ipiv)
{
    int info = 0;
    const float sfmin = FLT_MIN;
    for (int j = 0; j < imin(m, w); ++j) {
        int p = j;
        float best = fabsf(AT(A, lda, j, j));
        for (int i = j + 1; i < m; ++i) {
            float v = fabsf(AT(A, lda, i, j));
            if (v > best) { best = v; p = i; }
        }
        ipiv[j] = p + 1;
        float piv = AT(A, lda, p, j);
        if (piv != 0.0f) {
            if (p != j)
                for (int k = 0; k < w; ++k) {
                    float t = AT(A, lda, j, k);
                    AT(A, lda, j, k) = AT(A, lda, p, k);
                    AT(A, lda, p, k) = t;
                }
            if (fabsf(piv) >= sfmin) {
                float r = 1.0f / piv;
                for (int i = j + 1; i < m; ++i) AT(A, lda, i, j) *= r;
            } else {
                for (int i = j + 1; i < m; ++i) AT(A, lda, i, j) /= piv;
            }
        } else if (!info) {
            info = j + 1;
        }
        for (int k = j + 1; k < w; ++k) {
            float u = AT(A, lda, j, k);
            for (int i = j + 1; i < m; ++i) AT(A, lda, i, k) -= AT(A, lda, i, j) * u;
        }
    }
    return info;
}

/* apply_panel_pivots_kernel (src/getrf/getrf_pivot_kernels.hip:14-45):
 * swap rows in every column outside [panel, panel+size). */
static void apply_panel_pivots(float* A, int lda, int n, int panel, int size,
                               const int* local_piv)
{
    for (int c = 0; c < n; ++c) {
        if (c >= panel && c < panel + size) continue;
        for (int o = 0; o < size; ++o) {
            int r = panel + o, pr = panel + local_piv[o] - 1;
            if (pr != r) {
                float t = AT(A, lda, r, c);
                AT(A, lda, r, c) = AT(A, lda, pr, c);
                AT(A, lda, pr, c) = t;
            }
        }
    }
}

/*
 * Double-blocked left-looking LU with immediate pivots
 * (src/getrf/double_blocked_getrf.cpp:125-191), outer TRSM direct.
 * ipiv receives 1-based GLOBAL rows.
 */
int oracle_double_blocked_getrf(float* A, int lda, int n, int outer_nb,
                                int inner_nb, int* ipiv)
{
    int info = 0;
    if (n <= 0) return 0;
    if (outer_nb <= 0) outer_nb = n;
    if (inner_nb <= 0) inner_nb = outer_nb;
    inner_nb = imin(inner_nb, outer_nb);
    for (int outer = 0; outer < n; outer += outer_nb) {
        int outer_end = outer + imin(outer_nb, n - outer);
        for (int inner = outer; inner < outer_end; inner += inner_nb) {
            int isz = imin(inner_nb, outer_end - inner);
            int next = inner + isz;
            int f = getf2(n - inner, isz, &AT(A, lda, inner, inner), lda, ipiv + inner);
            if (f && !info) info = inner + f;
            apply_panel_pivots(A, lda, n, inner, isz, ipiv + inner);
            for (int o = 0; o < isz; ++o) ipiv[inner + o] += inner;
            if (next < outer_end) {
                int nsz = imin(inner_nb, outer_end - next);
                int hist = next - outer;
                trsm_left_lower_unit(hist, nsz, &AT(A, lda, outer, outer), lda,
                                     &AT(A, lda, outer, next), lda);
                gemm_nn_sub(n - next, nsz, hist, &AT(A, lda, next, outer), lda,
                            &AT(A, lda, outer, next), lda, &AT(A, lda, next, next), lda);
            }
        }
        if (outer_end < n) {
            int next = outer_end;
            int nsz = imin(outer_nb, n - next);
            trsm_left_lower_unit(next, nsz, A, lda, &AT(A, lda, 0, next), lda);
            gemm_nn_sub(n - next, nsz, next, &AT(A, lda, next, 0), lda,
                        &AT(A, lda, 0, next), lda, &AT(A, lda, next, next), lda);
        }
    }
    return info;
}
