/*
 * Body of the factor loops of factor.c, included once per scalar type with
 * REAL (the scalar), F(name) (the per-type function name), SQRT, FABS and
 * SFMIN (the smallest normal number, xGETF2's sfmin) defined.  TEST
 * INFRASTRUCTURE ONLY.
 */

/* LAPACK xPOTF2 (lower): returns 0 or the 1-based local failing column. */
static int F(potf2_lower)(int n, REAL* A, int lda)
{
    for (int j = 0; j < n; ++j) {
        REAL ajj = AT(A, lda, j, j);
        for (int k = 0; k < j; ++k) ajj -= AT(A, lda, j, k) * AT(A, lda, j, k);
        if (!(ajj > 0.0f)) {
            AT(A, lda, j, j) = ajj;
            return j + 1;
        }
        ajj = SQRT(ajj);
        AT(A, lda, j, j) = ajj;
        for (int i = j + 1; i < n; ++i) {
            REAL s = AT(A, lda, i, j);
            for (int k = 0; k < j; ++k) s -= AT(A, lda, i, k) * AT(A, lda, j, k);
            AT(A, lda, i, j) = s;
        }
        REAL r = 1.0f / ajj;
        for (int i = j + 1; i < n; ++i) AT(A, lda, i, j) *= r;
    }
    return 0;
}

/* B (rows x cols) <- B * L^{-T}, L lower non-unit cols x cols. */
static void F(trsm_right_lower_trans)(int rows, int cols, const REAL* L, int ldl,
                                   REAL* B, int ldb)
{
    for (int i = 0; i < rows; ++i) {
        for (int j = 0; j < cols; ++j) {
            REAL s = AT(B, ldb, i, j);
            for (int k = 0; k < j; ++k) s -= AT(B, ldb, i, k) * AT(L, ldl, j, k);
            AT(B, ldb, i, j) = s / AT(L, ldl, j, j);
        }
    }
}

/* C (rows x cols) -= A (rows x k) * B^T, B is cols x k. */
static void F(gemm_nt_sub)(int rows, int cols, int k, const REAL* A, int lda,
                        const REAL* B, int ldb, REAL* C, int ldc)
{
    for (int j = 0; j < cols; ++j)
        for (int p = 0; p < k; ++p) {
            REAL b = AT(B, ldb, j, p);
            for (int i = 0; i < rows; ++i) AT(C, ldc, i, j) -= AT(A, lda, i, p) * b;
        }
}

/* C_lower (n x n) -= A (n x k) * A^T. */
static void F(syrk_lower_sub)(int n, int k, const REAL* A, int lda, REAL* C, int ldc)
{
    for (int j = 0; j < n; ++j)
        for (int p = 0; p < k; ++p) {
            REAL b = AT(A, lda, j, p);
            for (int i = j; i < n; ++i) AT(C, ldc, i, j) -= AT(A, lda, i, p) * b;
        }
}

/* C (rows x cols) -= L (rows x k) * U (k x cols). */
static void F(gemm_nn_sub)(int rows, int cols, int k, const REAL* L, int ldl,
                        const REAL* U, int ldu, REAL* C, int ldc)
{
    for (int j = 0; j < cols; ++j)
        for (int p = 0; p < k; ++p) {
            REAL u = AT(U, ldu, p, j);
            for (int i = 0; i < rows; ++i) AT(C, ldc, i, j) -= AT(L, ldl, i, p) * u;
        }
}

/* B (rows x cols) <- L^{-1} B, L unit lower rows x rows. */
static void F(trsm_left_lower_unit)(int rows, int cols, const REAL* L, int ldl,
                                 REAL* B, int ldb)
{
    for (int j = 0; j < cols; ++j)
        for (int p = 0; p < rows; ++p) {
            REAL x = AT(B, ldb, p, j);
            for (int i = p + 1; i < rows; ++i) AT(B, ldb, i, j) -= AT(L, ldl, i, p) * x;
        }
}

/*
 * Double-blocked left-looking Cholesky, lower
 * (src/potrf/double_blocked_potrf.cpp:294-381).  nb<=0 -> n, b<=0 -> nb,
 * b = min(b, nb) (:309-321).  syrk_k_tile > 0 splits the outer SYRK's
 * reduction into chunks (src/syrk/kblocked_syrk.cpp:64-96).
 */
int F(oracle_double_blocked_potrf)(REAL* A, int lda, int n, int nb, int b,
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
            int f = F(potf2_lower)(isz, &AT(A, lda, inner, inner), lda);
            if (f && !info) info = inner + f;
            F(trsm_right_lower_trans)(n - ps, isz, &AT(A, lda, inner, inner), lda,
                                   &AT(A, lda, ps, inner), lda);
            if (ps < outer_end) {
                int pc = imin(b, outer_end - ps);
                /* full rectangle (rows ps..n) x (cols ps..ps+pc); the
                 * reference's GEMM also rewrites the diagonal block's strict
                 * upper triangle, which is never read back. */
                F(gemm_nt_sub)(n - ps, pc, ps - outer, &AT(A, lda, ps, outer), lda,
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
                F(syrk_lower_sub)(nsz, kc, &AT(A, lda, next, k0), lda,
                               &AT(A, lda, next, next), lda);
            }
            F(gemm_nt_sub)(n - below, nsz, next, &AT(A, lda, below, 0), lda,
                        &AT(A, lda, next, 0), lda, &AT(A, lda, below, next), lda);
        }
    }
    return info;
}

/*
 * LAPACK xGETF2 on an m x w panel: local 1-based pivots into ipiv[0..w),
 * returns 0 or the 1-based local column of the first exact zero pivot.
 */
static int F(getf2)(int m, int w, REAL* A, int lda, int* ipiv)
{
    int info = 0;
    const REAL sfmin = SFMIN;
    for (int j = 0; j < imin(m, w); ++j) {
        int p = j;
        REAL best = FABS(AT(A, lda, j, j));
        for (int i = j + 1; i < m; ++i) {
            REAL v = FABS(AT(A, lda, i, j));
            if (v > best) { best = v; p = i; }
        }
        ipiv[j] = p + 1;
        REAL piv = AT(A, lda, p, j);
        if (piv != 0.0f) {
            if (p != j)
                for (int k = 0; k < w; ++k) {
                    REAL t = AT(A, lda, j, k);
                    AT(A, lda, j, k) = AT(A, lda, p, k);
                    AT(A, lda, p, k) = t;
                }
            if (FABS(piv) >= sfmin) {
                REAL r = 1.0f / piv;
                for (int i = j + 1; i < m; ++i) AT(A, lda, i, j) *= r;
            } else {
                for (int i = j + 1; i < m; ++i) AT(A, lda, i, j) /= piv;
            }
        } else if (!info) {
            info = j + 1;
        }
        for (int k = j + 1; k < w; ++k) {
            REAL u = AT(A, lda, j, k);
            for (int i = j + 1; i < m; ++i) AT(A, lda, i, k) -= AT(A, lda, i, j) * u;
        }
    }
    return info;
}

/* apply_panel_pivots_kernel (src/getrf/getrf_pivot_kernels.hip:14-45):
 * swap rows in every column outside [panel, panel+size). */
static void F(apply_panel_pivots)(REAL* A, int lda, int n, int panel, int size,
                               const int* local_piv)
{
    for (int c = 0; c < n; ++c) {
        if (c >= panel && c < panel + size) continue;
        for (int o = 0; o < size; ++o) {
            int r = panel + o, pr = panel + local_piv[o] - 1;
            if (pr != r) {
                REAL t = AT(A, lda, r, c);
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
int F(oracle_double_blocked_getrf)(REAL* A, int lda, int n, int outer_nb,
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
            int f = F(getf2)(n - inner, isz, &AT(A, lda, inner, inner), lda, ipiv + inner);
            if (f && !info) info = inner + f;
            F(apply_panel_pivots)(A, lda, n, inner, isz, ipiv + inner);
            for (int o = 0; o < isz; ++o) ipiv[inner + o] += inner;
            if (next < outer_end) {
                int nsz = imin(inner_nb, outer_end - next);
                int hist = next - outer;
                F(trsm_left_lower_unit)(hist, nsz, &AT(A, lda, outer, outer), lda,
                                     &AT(A, lda, outer, next), lda);
                F(gemm_nn_sub)(n - next, nsz, hist, &AT(A, lda, next, outer), lda,
                            &AT(A, lda, outer, next), lda, &AT(A, lda, next, next), lda);
            }
        }
        if (outer_end < n) {
            int next = outer_end;
            int nsz = imin(outer_nb, n - next);
            F(trsm_left_lower_unit)(next, nsz, A, lda, &AT(A, lda, 0, next), lda);
            F(gemm_nn_sub)(n - next, nsz, next, &AT(A, lda, next, 0), lda,
                        &AT(A, lda, 0, next), lda, &AT(A, lda, next, next), lda);
        }
    }
    return info;
}

/* Rows r = k0..k1-1 of the LAPACK swap list ipiv (1-based GLOBAL rows) applied
 * in order to columns [c0, c0 + nc). */
static void F(swap_rows)(REAL* A, int lda, const int* ipiv, int k0, int k1, int c0, int nc)
{
    for (int c = c0; c < c0 + nc; ++c)
        for (int r = k0; r < k1; ++r) {
            int p = ipiv[r] - 1;
            if (p != r) {
                REAL t = AT(A, lda, r, c);
                AT(A, lda, r, c) = AT(A, lda, p, c);
                AT(A, lda, p, c) = t;
            }
        }
}

/*
 * Double-blocked left-looking LU with batched pivots
 * (src/getrf/getrf_batched_pivot_internal.h:445-624), outer TRSM direct:
 * after each panel its interchanges reach only the block's columns
 * ("inner pivot batch", :483-516); at the end of an outer block the block's
 * interchanges reach the earlier columns and every interchange so far reaches
 * the next block's columns ("outer pivot batch", :556-609), before that
 * block's outer TRSM + GEMM.  The host composition of the swaps into moved
 * rows (:59-223) is the same data movement as applying the swaps in order.
 * ipiv receives 1-based GLOBAL rows; the factors equal the immediate-pivot
 * loop's bit for bit.
 */
int F(oracle_double_blocked_getrf_batched)(REAL* A, int lda, int n, int outer_nb,
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
            int f = F(getf2)(n - inner, isz, &AT(A, lda, inner, inner), lda, ipiv + inner);
            if (f && !info) info = inner + f;
            for (int o = 0; o < isz; ++o) ipiv[inner + o] += inner;
            F(swap_rows)(A, lda, ipiv, inner, next, outer, inner - outer);
            F(swap_rows)(A, lda, ipiv, inner, next, next, outer_end - next);
            if (next < outer_end) {
                int nsz = imin(inner_nb, outer_end - next);
                int hist = next - outer;
                F(trsm_left_lower_unit)(hist, nsz, &AT(A, lda, outer, outer), lda,
                                        &AT(A, lda, outer, next), lda);
                F(gemm_nn_sub)(n - next, nsz, hist, &AT(A, lda, next, outer), lda,
                               &AT(A, lda, outer, next), lda, &AT(A, lda, next, next), lda);
            }
        }
        if (outer > 0) F(swap_rows)(A, lda, ipiv, outer, outer_end, 0, outer);
        if (outer_end < n) {
            int next = outer_end;
            int nsz = imin(outer_nb, n - next);
            F(swap_rows)(A, lda, ipiv, 0, outer_end, next, nsz);
            F(trsm_left_lower_unit)(next, nsz, A, lda, &AT(A, lda, 0, next), lda);
            F(gemm_nn_sub)(n - next, nsz, next, &AT(A, lda, next, 0), lda,
                           &AT(A, lda, 0, next), lda, &AT(A, lda, next, next), lda);
        }
    }
    return info;
}

/* LAPACK xGETF2 without row interchanges (the NPVT panels): returns 0 or the
 * 1-based local column of the first exact zero pivot. */
static int F(getf2_npvt)(int m, int w, REAL* A, int lda)
{
    int info = 0;
    const REAL sfmin = SFMIN;
    for (int j = 0; j < imin(m, w); ++j) {
        REAL piv = AT(A, lda, j, j);
        if (piv != 0.0f) {
            if (FABS(piv) >= sfmin) {
                REAL r = 1.0f / piv;
                for (int i = j + 1; i < m; ++i) AT(A, lda, i, j) *= r;
            } else {
                for (int i = j + 1; i < m; ++i) AT(A, lda, i, j) /= piv;
            }
        } else if (!info) {
            info = j + 1;
        }
        for (int k = j + 1; k < w; ++k) {
            REAL u = AT(A, lda, j, k);
            for (int i = j + 1; i < m; ++i) AT(A, lda, i, k) -= AT(A, lda, i, j) * u;
        }
    }
    return info;
}

/*
 * Blocked right-looking Cholesky, lower (src/potrf/blocked_potrf.cpp:127-181):
 * per block column potf2 on the diagonal block, the panel TRSM and the lower
 * SYRK of the whole trailing matrix.
 */
int F(oracle_blocked_right_looking_potrf)(REAL* A, int lda, int n, int nb)
{
    int info = 0;
    if (n <= 0) return 0;
    if (nb <= 0) nb = n;
    for (int k = 0; k < n; k += nb) {
        int psz = imin(nb, n - k);
        int tr = n - k - psz;
        int f = F(potf2_lower)(psz, &AT(A, lda, k, k), lda);
        if (f && !info) info = k + f;
        if (tr <= 0) continue;
        F(trsm_right_lower_trans)(tr, psz, &AT(A, lda, k, k), lda, &AT(A, lda, k + psz, k), lda);
        F(syrk_lower_sub)(tr, psz, &AT(A, lda, k + psz, k), lda, &AT(A, lda, k + psz, k + psz),
                          lda);
    }
    return info;
}

/*
 * Blocked right-looking LU (src/getrf/blocked_getrf.cpp:15-71; pivot = 0 gives
 * the NPVT variant, src/getrf/blocked_getrf_npvt.cpp): panel GETF2 over the
 * remaining rows, its interchanges on every other column, the U12 TRSM and
 * the trailing GEMM.  ipiv (1-based GLOBAL rows) is written when pivoting.
 */
int F(oracle_blocked_right_looking_getrf)(REAL* A, int lda, int n, int nb, int* ipiv,
                                          int pivot)
{
    int info = 0;
    if (n <= 0) return 0;
    if (nb <= 0) nb = n;
    for (int p = 0; p < n; p += nb) {
        int psz = imin(nb, n - p);
        int next = p + psz;
        int tr = n - next;
        int f;
        if (pivot) {
            f = F(getf2)(n - p, psz, &AT(A, lda, p, p), lda, ipiv + p);
            F(apply_panel_pivots)(A, lda, n, p, psz, ipiv + p);
            for (int o = 0; o < psz; ++o) ipiv[p + o] += p;
        } else {
            f = F(getf2_npvt)(n - p, psz, &AT(A, lda, p, p), lda);
        }
        if (f && !info) info = p + f;
        if (tr <= 0) continue;
        F(trsm_left_lower_unit)(psz, tr, &AT(A, lda, p, p), lda, &AT(A, lda, p, next), lda);
        F(gemm_nn_sub)(tr, tr, psz, &AT(A, lda, next, p), lda, &AT(A, lda, p, next), lda,
                       &AT(A, lda, next, next), lda);
    }
    return info;
}

/*
 * Recursive Cholesky, lower (src/potrf/recursive_potrf.cpp:17-174): below
 * order nb the diagonal POTRF; above it the split n1 = n/2, POTRF(A11),
 * A21 <- A21 L11^{-T}, A22 -= A21 A21^T, POTRF(A22).  info is global.
 */
static int F(rec_potrf)(REAL* A, int lda, int n, int nb, int base)
{
    if (n <= 0) return 0;
    if (nb <= 0 || n <= nb) {
        int f = F(potf2_lower)(n, A, lda);
        return f ? base + f : 0;
    }
    int n1 = n / 2, n2 = n - n1;
    int info = F(rec_potrf)(A, lda, n1, nb, base);
    if (info) return info;
    F(trsm_right_lower_trans)(n2, n1, A, lda, &AT(A, lda, n1, 0), lda);
    F(syrk_lower_sub)(n2, n1, &AT(A, lda, n1, 0), lda, &AT(A, lda, n1, n1), lda);
    return F(rec_potrf)(&AT(A, lda, n1, n1), lda, n2, nb, base + n1);
}

int F(oracle_recursive_potrf)(REAL* A, int lda, int n, int nb)
{
    return F(rec_potrf)(A, lda, n, nb, 0);
}
