/*
 * CPU FP64 residual oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference's host residual harness
 * (include/utils/benchmark/cpu_fp64_residual.h).  Only tests, the smoke check
 * and the CPU-baseline leg of bench.py may load this file's library; the
 * product path (the CUDA library) never calls into it.
 *
 * What it computes (cpu_fp64_residual.h:73-139):
 *   ||A - L L^T||_F / ||A||_F            (Cholesky, lower factor)
 *   ||P A - L U||_F / ||A||_F            (LU, packed unit-lower L and upper U)
 * with every stored FP32/FP64 value widened to double BEFORE it is multiplied,
 * products accumulated in FP64 over bounded tiles, structurally zero triangular
 * products skipped (k > min(row, column)), and both Frobenius norms formed with
 * an overflow-safe scaled sum of squares (cpu_fp64_residual.h:29-50).
 *
 * Edge-case contract, identical to the reference (test_cpu_fp64_residual.cpp):
 *   - non-finite value anywhere  -> +inf
 *   - 0/0 -> 0,  x/0 -> +inf
 *   - invalid LU pivot (ipiv[r] < r+1 or > n) -> +inf   (cpu_fp64_residual.h:157-163)
 *   - n <= 0, lda < n, tile <= 0, null pointers -> *err = 1 (the reference throws
 *     std::invalid_argument, cpu_fp64_residual.h:79-81, 150-153, 185-188)
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double scale;
    double sum;
    int finite;
} ssq_t;

/* cpu_fp64_residual.h:29-50 -- scaled sum of squares. */
static void ssq_add(ssq_t* s, double v)
{
    double m = fabs(v);
    if (!isfinite(m)) {
        s->finite = 0;
    } else if (m != 0.0) {
        if (s->scale < m) {
            double r = s->scale / m;
            s->sum = 1.0 + s->sum * r * r;
            s->scale = m;
        } else {
            double r = m / s->scale;
            s->sum += r * r;
        }
    }
}

static double ssq_ratio(const ssq_t* num, const ssq_t* den)
{
    /* cpu_fp64_residual.h:130-138 */
    if (!num->finite || !den->finite) return INFINITY;
    if (den->scale == 0.0) return num->scale == 0.0 ? 0.0 : INFINITY;
    return (num->scale / den->scale) * sqrt(num->sum / den->sum);
}

/* Element accessors: kind 0 = Cholesky (lower L), kind 1 = LU (packed). */
typedef struct {
    int kind;
    int is_double;
    const void* factor;
    const void* original;
    const int* perm; /* row permutation for LU (NULL = identity) */
    size_t lda;
} access_t;

static inline double load(const void* p, int is_double, size_t idx)
{
    return is_double ? ((const double*)p)[idx] : (double)((const float*)p)[idx];
}

/* left(row, k): L(row, k) */
static inline double left_at(const access_t* a, int row, int k)
{
    if (row < k) return 0.0;
    if (a->kind == 1 && row == k) return 1.0;
    return load(a->factor, a->is_double, (size_t)k * a->lda + row);
}

/* right(k, col): L^T(k, col) = L(col, k) for Cholesky, U(k, col) for LU */
static inline double right_at(const access_t* a, int k, int col)
{
    if (a->kind == 0) {
        if (col < k) return 0.0;
        return load(a->factor, a->is_double, (size_t)k * a->lda + col);
    }
    if (k > col) return 0.0;
    return load(a->factor, a->is_double, (size_t)col * a->lda + k);
}

static inline double original_at(const access_t* a, int row, int col)
{
    int r = a->perm ? a->perm[row] : row;
    return load(a->original, a->is_double, (size_t)col * a->lda + r);
}

/*
 * Tiled FP64 product with structural-zero skipping
 * (cpu_fp64_residual.h:92-128): each (row tile, column tile) accumulates the
 * full reduction up to min(row_end, col_end), then contributes to both norms.
 */
static double full_residual(int n, int tile, const access_t* a)
{
    if (tile > n) tile = n;
    size_t cap = (size_t)tile * (size_t)tile;
    double* lt = (double*)malloc(cap * sizeof(double));
    double* rt = (double*)malloc(cap * sizeof(double));
    double* pr = (double*)malloc(cap * sizeof(double));
    ssq_t res = {0.0, 1.0, 1};
    ssq_t org = {0.0, 1.0, 1};
    if (!lt || !rt || !pr) {
        free(lt); free(rt); free(pr);
        return NAN;
    }
    for (int c0 = 0; c0 < n; c0 += tile) {
        int nc = (n - c0 < tile) ? n - c0 : tile;
        for (int r0 = 0; r0 < n; r0 += tile) {
            int nr = (n - r0 < tile) ? n - r0 : tile;
            memset(pr, 0, (size_t)nr * nc * sizeof(double));
            int kend = (r0 + nr < c0 + nc) ? r0 + nr : c0 + nc;
            for (int k0 = 0; k0 < kend; k0 += tile) {
                int nk = (kend - k0 < tile) ? kend - k0 : tile;
                for (int k = 0; k < nk; ++k)
                    for (int i = 0; i < nr; ++i)
                        lt[(size_t)k * nr + i] = left_at(a, r0 + i, k0 + k);
                for (int j = 0; j < nc; ++j)
                    for (int k = 0; k < nk; ++k)
                        rt[(size_t)j * nk + k] = right_at(a, k0 + k, c0 + j);
                for (int j = 0; j < nc; ++j) {
                    double* pc = pr + (size_t)j * nr;
                    for (int k = 0; k < nk; ++k) {
                        double v = rt[(size_t)j * nk + k];
                        const double* lc = lt + (size_t)k * nr;
                        for (int i = 0; i < nr; ++i) pc[i] += lc[i] * v;
                    }
                }
            }
            for (int j = 0; j < nc; ++j) {
                for (int i = 0; i < nr; ++i) {
                    double o = original_at(a, r0 + i, c0 + j);
                    ssq_add(&org, o);
                    ssq_add(&res, pr[(size_t)j * nr + i] - o);
                }
            }
        }
    }
    free(lt); free(rt); free(pr);
    return ssq_ratio(&res, &org);
}

static double potrf_residual(const void* L, const void* A, int n, int lda,
                             int tile, int is_double, int* err)
{
    *err = 0;
    if (n <= 0 || lda < n || tile <= 0 || !L || !A) { *err = 1; return NAN; }
    access_t a = {0, is_double, L, A, NULL, (size_t)lda};
    return full_residual(n, tile, &a);
}

static double getrf_residual(const void* LU, const void* A, const int* ipiv,
                             int n, int lda, int pivoting, int tile,
                             int is_double, int* err)
{
    *err = 0;
    if (n <= 0 || lda < n || tile <= 0 || !LU || !A || (pivoting && !ipiv)) {
        *err = 1;
        return NAN;
    }
    int* perm = (int*)malloc((size_t)n * sizeof(int));
    if (!perm) { *err = 2; return NAN; }
    for (int i = 0; i < n; ++i) perm[i] = i;
    if (pivoting) {
        /* One-based global LAPACK pivots applied in order
         * (cpu_fp64_residual.h:156-164). */
        for (int r = 0; r < n; ++r) {
            int p = ipiv[r];
            if (p < r + 1 || p > n) { free(perm); return INFINITY; }
            int t = perm[r]; perm[r] = perm[p - 1]; perm[p - 1] = t;
        }
    }
    access_t a = {1, is_double, LU, A, perm, (size_t)lda};
    double r = full_residual(n, tile, &a);
    free(perm);
    return r;
}

double oracle_potrf_residual_f32(const float* L, const float* A, int n, int lda,
                                 int tile, int* err)
{
    return potrf_residual(L, A, n, lda, tile, 0, err);
}

double oracle_potrf_residual_f64(const double* L, const double* A, int n, int lda,
                                 int tile, int* err)
{
    return potrf_residual(L, A, n, lda, tile, 1, err);
}

double oracle_getrf_residual_f32(const float* LU, const float* A, const int* ipiv,
                                 int n, int lda, int pivoting, int tile, int* err)
{
    return getrf_residual(LU, A, ipiv, n, lda, pivoting, tile, 0, err);
}

double oracle_getrf_residual_f64(const double* LU, const double* A, const int* ipiv,
                                 int n, int lda, int pivoting, int tile, int* err)
{
    return getrf_residual(LU, A, ipiv, n, lda, pivoting, tile, 1, err);
}

/*
 * Seed parser, restating include/utils/benchmark/seed.h:5-19: decimal digits
 * only, no sign, rejects overflow past UINT32_MAX; leaves *seed untouched on
 * failure.
 */
int oracle_parse_seed(const char* text, unsigned int* seed)
{
    if (text == NULL || *text == '\0') return 0;
    unsigned int v = 0;
    for (const char* d = text; *d; ++d) {
        if (*d < '0' || *d > '9') return 0;
        unsigned int next = (unsigned int)(*d - '0');
        if (v > (0xFFFFFFFFu - next) / 10u) return 0;
        v = v * 10u + next;
    }
    *seed = v;
    return 1;
}
