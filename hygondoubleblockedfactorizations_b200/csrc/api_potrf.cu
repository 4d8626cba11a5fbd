// C ABI: Cholesky drivers and the SYRK / TRSM / GEMM entry points.
//
// Every function mirrors the reference signature (with hdbf_handle in place
// of rocblas_handle), records its status in the handle and never exits.
#include <algorithm>

#include "internal.h"
#include "gemm/update_gemm.h"
#include "potrf/blocked_potrf.h"
#include "potrf/double_blocked_potrf.h"
#include "potrf/recursive_potrf.h"
#include "syrk/batched_syrk.h"
#include "syrk/kblocked_syrk.h"
#include "syrk/recursive_syrk.h"
#include "trsm/double_blocked_trsm.h"
#include "trsm/iterative_trsm.h"
#include "trsm/recursive_trsm.h"
#include "trsm/right_lower_trsm.h"

namespace hdbf {
namespace {

// Reference tuning constants (src/potrf/double_blocked_potrf.cpp:17-20,
// src/trsm/recursive_trsm.cpp:12).
constexpr int kPotrfDbTrsmMicroBlock = 1024;
constexpr int kInnerGemmMTile = 8192;
constexpr int kInnerGemmMThreshold = 32768;
constexpr int kInnerGemmKThreshold = 5632;
constexpr int kTrsmUpdateTile = 8192;

template <class T>
inline T* at(T* A, long long lda, int r, int c) { return A + (long long)c * lda + r; }

hdbf_status record(hdbf_context* ctx, hdbf_status st)
{
    if (ctx) ctx->last_status = st;
    return st;
}

bool bad_matrix(const void* A, int lda, int rows)
{
    return rows < 0 || (rows > 0 && (!A || lda < std::max(1, rows)));
}

// C(rows x cols) -= A * B^T in row chunks of m_tile (<=0: one pass).  When
// `diag_first` the top cols x cols block of C is a diagonal block: only its
// lower triangle is updated.
template <class T>
hdbf_status gemm_nt_rows(hdbf_context* ctx, int rows, int cols, int k, const T* A,
                         long long lda, const T* B, long long ldb, T* C,
                         long long ldc, int m_tile, bool diag_first)
{
    if (rows <= 0 || cols <= 0 || k <= 0) return HDBF_STATUS_SUCCESS;
    int r = 0;
    if (diag_first) {
        // One lower-trapezoid launch covers the diagonal block and the rows
        // below it (of the first M tile), so the small diagonal block does not
        // run as a separate, mostly idle launch.  Each entry is the same k-order
        // sum either way.
        const int first = std::min(rows, std::max(cols, m_tile > 0 ? m_tile : rows));
        HDBF_TRY(gemm_sub(ctx, false, true, first, cols, k, A, lda, B, ldb, C, ldc));
        r = first;
    }
    const int tile = m_tile > 0 ? m_tile : rows;
    for (; r < rows; r += tile) {
        const int tr = std::min(tile, rows - r);
        HDBF_TRY(gemm_sub(ctx, false, false, tr, cols, k, A + r, lda, B, ldb, C + r, ldc));
    }
    return HDBF_STATUS_SUCCESS;
}

// src/trsm/double_blocked_trsm.cpp:99-171: B (n x m) <- B * L^{-T}.
template <class T>
hdbf_status dbtrsm_impl(hdbf_context* ctx, const T* L, long long ldl, T* B,
                        long long ldb, int n, int m, int nb, int b)
{
    if (n <= 0 || m <= 0) return HDBF_STATUS_SUCCESS;
    if (nb <= 0) nb = m;
    if (b <= 0) b = nb;
    b = std::min(b, nb);
    for (int outer = 0; outer < m; outer += nb) {
        const int osz = std::min(nb, m - outer);
        const int oend = outer + osz;
        for (int inner = outer; inner < oend; inner += b) {
            const int isz = std::min(b, oend - inner);
            const int ps = inner + isz;
            HDBF_TRY(trsm_rlt(ctx, n, isz, at(L, ldl, inner, inner), ldl, at(B, ldb, 0, inner), ldb));
            if (ps < oend) {
                const int pc = std::min(b, oend - ps);
                HDBF_TRY(gemm_sub(ctx, false, false, n, pc, ps - outer, at(B, ldb, 0, outer), ldb,
                                   at(L, ldl, ps, outer), ldl, at(B, ldb, 0, ps), ldb));
            }
        }
        const int trailing = m - oend;
        if (trailing > 0)
            HDBF_TRY(gemm_sub(ctx, false, false, n, trailing, osz, at(B, ldb, 0, outer), ldb,
                               at(L, ldl, oend, outer), ldl, at(B, ldb, 0, oend), ldb));
    }
    return HDBF_STATUS_SUCCESS;
}

// src/potrf/double_blocked_potrf.cpp:294-381 with this library's kernels.
template <class T>
hdbf_status potrf_db_impl(hdbf_context* ctx, T* A, int lda, int n, int nb, int b, int* info,
                          bool use_dbtrsm, int syrk_k_tile, int m_tile, int m_thr, int k_thr)
{
    if (bad_matrix(A, lda, n)) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0) {
        if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
        return last_cuda(ctx);
    }
    HDBF_TRY(ensure_ws(ctx, ws_order<T>(n)));
    if (nb <= 0) nb = n;
    if (b <= 0) b = nb;
    b = std::min(b, nb);
    const std::vector<long long> key = {1 + type_tag<T>(), (long long)A, lda, n, nb, b, (long long)info,
                                        use_dbtrsm, syrk_k_tile, m_tile, m_thr, k_thr};
    return run_graph(ctx, key, [&]() -> hdbf_status {
    if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
    for (int outer = 0; outer < n; outer += nb) {
        const int oend = outer + std::min(nb, n - outer);
        for (int inner = outer; inner < oend; inner += b) {
            const int isz = std::min(b, oend - inner);
            const int ps = inner + isz;
            const int rows = n - ps;
            T* Aii = at(A, lda, inner, inner);
            {
                StageScope sc(ctx, kStPotrf);
                HDBF_TRY(potrf_diag(ctx, isz, Aii, lda, info, inner));
            }
            {
                StageScope sc(ctx, kStTrsm);
                if (use_dbtrsm) {
                    HDBF_TRY(dbtrsm_impl(ctx, Aii, lda, at(A, lda, ps, inner), lda, rows, isz,
                                         isz, std::min(kPotrfDbTrsmMicroBlock, isz)));
                } else {
                    HDBF_TRY(trsm_rlt(ctx, rows, isz, Aii, lda, at(A, lda, ps, inner), lda));
                }
            }
            if (ps < oend) {  // update_next_inner_panel (:210-249)
                StageScope sc(ctx, kStInnerGemm);
                const int pc = std::min(b, oend - ps);
                const int k = ps - outer;
                const bool mt = m_tile > 0 && rows > m_thr && k >= k_thr;
                HDBF_TRY(gemm_nt_rows(ctx, rows, pc, k, at(A, lda, ps, outer), lda,
                                      at(A, lda, ps, outer), lda, at(A, lda, ps, ps), lda,
                                      mt ? m_tile : 0, true));
            }
        }
        if (oend < n) {  // prepare_next_outer_panel (:251-292)
            const int next = oend;
            const int nsz = std::min(nb, n - next);
            const int below = next + nsz;
            const int tk = (syrk_k_tile > 0 && syrk_k_tile < next) ? syrk_k_tile : next;
            if (tk == next) {
                // Unblocked K: the SYRK of the next diagonal block and the
                // GEMM below it share both operands and K, so one
                // lower-trapezoid launch does both (same per-entry sums).
                StageScope sc(ctx, kStOuterGemm);
                HDBF_TRY(gemm_nt_rows(ctx, n - next, nsz, next, at(A, lda, next, 0), lda,
                                      at(A, lda, next, 0), lda, at(A, lda, next, next), lda, 0,
                                      true));
                continue;
            }
            {
                StageScope sc(ctx, kStOuterSyrk);
                for (int k0 = 0; k0 < next; k0 += tk) {
                    const int kc = std::min(tk, next - k0);
                    HDBF_TRY(syrk_lower(ctx, nsz, kc, at(A, lda, next, k0), lda,
                                        at(A, lda, next, next), lda));
                }
            }
            StageScope sc(ctx, kStOuterGemm);
            HDBF_TRY(gemm_sub(ctx, false, false, n - below, nsz, next, at(A, lda, below, 0), lda,
                               at(A, lda, next, 0), lda, at(A, lda, below, next), lda));
        }
    }
    return last_cuda(ctx);
    });
}

// src/potrf/blocked_potrf.cpp:126-178.
template <class T>
hdbf_status potrf_blocked_rl_impl(hdbf_context* ctx, T* A, int lda, int n, int nb, int* info)
{
    if (bad_matrix(A, lda, n)) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0) {
        if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
        return last_cuda(ctx);
    }
    HDBF_TRY(ensure_ws(ctx, ws_order<T>(n)));
    if (nb <= 0) nb = n;
    const std::vector<long long> key = {2 + type_tag<T>(), (long long)A, lda, n, nb, (long long)info};
    return run_graph(ctx, key, [&]() -> hdbf_status {
    if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
    for (int k = 0; k < n; k += nb) {
        const int psz = std::min(nb, n - k);
        const int tr = n - k - psz;
        T* Akk = at(A, lda, k, k);
        HDBF_TRY(potrf_diag(ctx, psz, Akk, lda, info, k));
        if (tr <= 0) continue;
        T* A21 = at(A, lda, k + psz, k);
        HDBF_TRY(trsm_rlt(ctx, tr, psz, Akk, lda, A21, lda));
        HDBF_TRY(syrk_lower(ctx, tr, psz, A21, lda, at(A, lda, k + psz, k + psz), lda));
    }
    return last_cuda(ctx);
    });
}

// src/trsm/recursive_trsm.cpp:132-200: B (n x m) <- B * L^{-T}, split m.
template <class T>
hdbf_status rec_trsm_impl(hdbf_context* ctx, const T* L, long long ldl, T* B,
                          long long ldb, int n, int m, int nb, bool tiled)
{
    if (n <= 0 || m <= 0) return HDBF_STATUS_SUCCESS;
    if (m <= nb || nb <= 0) return trsm_rlt(ctx, n, m, L, ldl, B, ldb);
    const int m1 = m / 2;
    const int m2 = m - m1;
    HDBF_TRY(rec_trsm_impl(ctx, L, ldl, B, ldb, n, m1, nb, tiled));
    // B2 -= X1 * L21^T, optionally tiled 8192 x 8192 x 8192 (:82-122)
    const int t = tiled ? kTrsmUpdateTile : std::max(std::max(n, m1), m2);
    for (int r = 0; r < n; r += t)
        for (int c = 0; c < m2; c += t)
            for (int kk = 0; kk < m1; kk += t)
                HDBF_TRY(gemm_sub(ctx, false, false, std::min(t, n - r), std::min(t, m2 - c),
                                   std::min(t, m1 - kk), at(B, ldb, r, kk), ldb,
                                   at(L, ldl, m1 + c, kk), ldl, at(B, ldb, r, m1 + c), ldb));
    return rec_trsm_impl(ctx, at(L, ldl, m1, m1), ldl, at(B, ldb, 0, m1), ldb, n, m2, nb, tiled);
}

// C_lower -= A A^T as nb x nb diagonal leaves plus off-diagonal block rows
// (src/syrk/batched_syrk.cpp:27-153).
template <class T>
hdbf_status batched_syrk_impl(hdbf_context* ctx, const T* A, long long lda, T* C,
                              long long ldc, int n, int k, int nb)
{
    if (n <= 0 || k <= 0) return HDBF_STATUS_SUCCESS;
    if (nb <= 0 || nb >= n) return syrk_lower(ctx, n, k, A, lda, C, ldc);
    for (int i = 0; i < n; i += nb) {
        const int bs = std::min(nb, n - i);
        HDBF_TRY(syrk_lower(ctx, bs, k, A + i, lda, at(C, ldc, i, i), ldc));
        if (i > 0)
            HDBF_TRY(gemm_sub(ctx, false, false, bs, i, k, A + i, lda, A, lda, C + i, ldc));
    }
    return HDBF_STATUS_SUCCESS;
}

// src/syrk/recursive_syrk.cpp:9-45.
template <class T>
hdbf_status rec_syrk_impl(hdbf_context* ctx, const T* A, long long lda, T* C,
                          long long ldc, int n, int k, int nb)
{
    if (n <= 0 || k <= 0) return HDBF_STATUS_SUCCESS;
    if (nb <= 0 || n <= nb) return syrk_lower(ctx, n, k, A, lda, C, ldc);
    const int n1 = n / 2;
    const int n2 = n - n1;
    HDBF_TRY(rec_syrk_impl(ctx, A, lda, C, ldc, n1, k, nb));
    HDBF_TRY(gemm_sub(ctx, false, false, n2, n1, k, A + n1, lda, A, lda, C + n1, ldc));
    return rec_syrk_impl(ctx, A + n1, lda, at(C, ldc, n1, n1), ldc, n2, k, nb);
}

// src/potrf/recursive_potrf.cpp:17-174.
template <class T>
hdbf_status rec_potrf_impl(hdbf_context* ctx, T* A, long long lda, int n, int nb, int* info,
                           int info_base, bool tiled)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    if (nb <= 0 || n <= nb) return potrf_diag(ctx, n, A, lda, info, info_base);
    const int n1 = n / 2;
    const int n2 = n - n1;
    T* A21 = A + n1;
    T* A22 = at(A, lda, n1, n1);
    HDBF_TRY(rec_potrf_impl(ctx, A, lda, n1, nb, info, info_base, tiled));
    HDBF_TRY(rec_trsm_impl(ctx, A, lda, A21, lda, n2, n1, nb, tiled));
    HDBF_TRY(batched_syrk_impl(ctx, A21, lda, A22, lda, n2, n1, nb));
    return rec_potrf_impl(ctx, A22, lda, n2, nb, info, info_base + n1, tiled);
}

template <class T>
hdbf_status rec_potrf_entry(hdbf_context* ctx, T* A, int lda, int n, int nb, int* info,
                            bool tiled)
{
    if (bad_matrix(A, lda, n)) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0) {
        if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
        return last_cuda(ctx);
    }
    HDBF_TRY(ensure_ws(ctx, ws_order<T>(n)));
    const std::vector<long long> key = {3 + type_tag<T>(), (long long)A, lda, n, nb, (long long)info, tiled};
    return run_graph(ctx, key, [&]() -> hdbf_status {
        if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
        HDBF_TRY(rec_potrf_impl(ctx, A, lda, n, nb, info, 0, tiled));
        return last_cuda(ctx);
    });
}

}  // namespace
}  // namespace hdbf

using namespace hdbf;

#define HDBF_ABI(handle, expr)                 \
    do {                                       \
        if (!(handle)) return;                 \
        record((handle), (expr));              \
    } while (0)

extern "C" {

void double_blocked_potrf(hdbf_handle h, float* A, int lda, int n, int nb, int b, int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, 0, 0, 0, 0));
}

void double_blocked_potrf_dbtrsm(hdbf_handle h, float* A, int lda, int n, int nb, int b,
                                 int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, true, 0, 0, 0, 0));
}

void double_blocked_potrf_kblocked_syrk(hdbf_handle h, float* A, int lda, int n, int nb, int b,
                                        int syrk_k_tile, int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, syrk_k_tile, 0, 0, 0));
}

void double_blocked_potrf_kblocked_syrk_adaptive_gemm(hdbf_handle h, float* A, int lda, int n,
                                                      int nb, int b, int syrk_k_tile, int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, syrk_k_tile, kInnerGemmMTile,
                              kInnerGemmMThreshold, kInnerGemmKThreshold));
}

void double_blocked_potrf_kblocked_syrk_adaptive_gemm_configured(
    hdbf_handle h, float* A, int lda, int n, int nb, int b, int syrk_k_tile, int gemm_m_tile,
    int gemm_m_threshold, int gemm_k_threshold, int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, syrk_k_tile, gemm_m_tile,
                              gemm_m_threshold, gemm_k_threshold));
}

void blocked_right_looking_potrf(hdbf_handle h, float* A, int lda, int n, int nb, int* info)
{
    HDBF_ABI(h, potrf_blocked_rl_impl(h, A, lda, n, nb, info));
}

void recursive_potrf(hdbf_handle h, StreamPool* pool, float* A, int lda, int n, int nb,
                     int* info)
{
    (void)pool;
    if (!h) return;
    record(h, rec_potrf_entry(h, A, lda, n, nb, info, false));
}

void recursive_potrf_tiled_trsm(hdbf_handle h, StreamPool* pool, float* A, int lda, int n,
                                int nb, int* info)
{
    (void)pool;
    if (!h) return;
    record(h, rec_potrf_entry(h, A, lda, n, nb, info, true));
}

void syrk_lower_update(hdbf_handle h, int n, int k, const float* A, int lda, float* C, int ldc)
{
    HDBF_ABI(h, syrk_lower(h, n, k, A, lda, C, ldc));
}

void syrk_lower_update_kblocked(hdbf_handle h, int n, int k, const float* A, int lda, float* C,
                                int ldc, int k_tile)
{
    if (!h) return;
    if (n <= 0 || k <= 0) { record(h, HDBF_STATUS_SUCCESS); return; }
    const int tk = (k_tile <= 0 || k_tile >= k) ? k : k_tile;
    hdbf_status st = HDBF_STATUS_SUCCESS;
    for (int k0 = 0; k0 < k && st == HDBF_STATUS_SUCCESS; k0 += tk)
        st = syrk_lower(h, n, std::min(tk, k - k0), A + (long long)k0 * lda, lda, C, ldc);
    record(h, st);
}

void recursive_syrk_parallel(hdbf_handle h, float* A, int lda, float* C, int ldc, int n, int k,
                             int nb)
{
    HDBF_ABI(h, rec_syrk_impl(h, A, lda, C, ldc, n, k, nb));
}

void batched_syrk_bottom_up(hdbf_handle h, StreamPool* pool, float* A, int lda, float* C,
                            int ldc, int n, int k, int nb)
{
    (void)pool;
    HDBF_ABI(h, batched_syrk_impl(h, A, lda, C, ldc, n, k, nb));
}

void trsm_right_lower_transpose(hdbf_handle h, int rows, int cols, const float* A, int lda,
                                float* B, int ldb)
{
    HDBF_ABI(h, trsm_rlt(h, rows, cols, A, lda, B, ldb));
}

void double_blocked_trsm(hdbf_handle h, float* A, int lda, float* B, int ldb, int n, int m,
                         int nb, int b)
{
    HDBF_ABI(h, dbtrsm_impl(h, A, lda, B, ldb, n, m, nb, b));
}

void recursive_trsm(hdbf_handle h, float* A, int lda, float* B, int ldb, int n, int m, int nb)
{
    HDBF_ABI(h, rec_trsm_impl(h, A, lda, B, ldb, n, m, nb, false));
}

void recursive_trsm_tiled_update(hdbf_handle h, float* A, int lda, float* B, int ldb, int n,
                                 int m, int nb)
{
    HDBF_ABI(h, rec_trsm_impl(h, A, lda, B, ldb, n, m, nb, true));
}

void iterative_trsm_right_looking(hdbf_handle h, float* A, int lda, float* B, int ldb, int n,
                                  int m, int nb)
{
    if (!h) return;
    if (n <= 0 || m <= 0) { record(h, HDBF_STATUS_SUCCESS); return; }
    if (nb <= 0) nb = m;
    hdbf_status st = HDBF_STATUS_SUCCESS;
    // src/trsm/iterative_trsm.cpp:18-56
    for (int i = 0; i < m && st == HDBF_STATUS_SUCCESS; i += nb) {
        const int cur = std::min(nb, m - i);
        st = trsm_rlt(h, n, cur, at(A, lda, i, i), lda, at(B, ldb, 0, i), ldb);
        if (st == HDBF_STATUS_SUCCESS && i + cur < m)
            st = sgemm_sub(h, false, false, n, m - i - cur, cur, at(B, ldb, 0, i), ldb,
                           at(A, lda, i + cur, i), lda, at(B, ldb, 0, i + cur), ldb);
    }
    record(h, st);
}

void gemm_nt_update(hdbf_handle h, int rows, int cols, int k, const float* A, int lda,
                    const float* B, int ldb, float* C, int ldc)
{
    HDBF_ABI(h, sgemm_sub(h, false, false, rows, cols, k, A, lda, B, ldb, C, ldc));
}

void gemm_nt_update_m_tiled(hdbf_handle h, int rows, int cols, int k, const float* A, int lda,
                            const float* B, int ldb, float* C, int ldc, int m_tile)
{
    HDBF_ABI(h, gemm_nt_rows(h, rows, cols, k, A, lda, B, ldb, C, ldc, m_tile, false));
}

// ------------------------------------------------------------ FP64 twins
// The reference's `_double` entry points: the same drivers instantiated for
// double on this library's FP64 kernels (fp64.cu).

void double_blocked_potrf_double(hdbf_handle h, double* A, int lda, int n, int nb, int b,
                                 int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, 0, 0, 0, 0));
}

void double_blocked_potrf_double_dbtrsm(hdbf_handle h, double* A, int lda, int n, int nb, int b,
                                        int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, true, 0, 0, 0, 0));
}

void double_blocked_potrf_double_kblocked_syrk(hdbf_handle h, double* A, int lda, int n, int nb,
                                               int b, int syrk_k_tile, int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, syrk_k_tile, 0, 0, 0));
}

void double_blocked_potrf_double_kblocked_syrk_adaptive_gemm(hdbf_handle h, double* A, int lda,
                                                             int n, int nb, int b,
                                                             int syrk_k_tile, int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, syrk_k_tile, kInnerGemmMTile,
                              kInnerGemmMThreshold, kInnerGemmKThreshold));
}

void double_blocked_potrf_double_kblocked_syrk_adaptive_gemm_configured(
    hdbf_handle h, double* A, int lda, int n, int nb, int b, int syrk_k_tile, int gemm_m_tile,
    int gemm_m_threshold, int gemm_k_threshold, int* info)
{
    HDBF_ABI(h, potrf_db_impl(h, A, lda, n, nb, b, info, false, syrk_k_tile, gemm_m_tile,
                              gemm_m_threshold, gemm_k_threshold));
}

void blocked_right_looking_potrf_double(hdbf_handle h, double* A, int lda, int n, int nb,
                                        int* info)
{
    HDBF_ABI(h, potrf_blocked_rl_impl(h, A, lda, n, nb, info));
}

void recursive_potrf_double(hdbf_handle h, StreamPool* pool, double* A, int lda, int n, int nb,
                            int* info)
{
    (void)pool;
    if (!h) return;
    record(h, rec_potrf_entry(h, A, lda, n, nb, info, false));
}

void syrk_lower_update_double(hdbf_handle h, int n, int k, const double* A, int lda, double* C,
                              int ldc)
{
    HDBF_ABI(h, syrk_lower(h, n, k, A, lda, C, ldc));
}

void syrk_lower_update_kblocked_double(hdbf_handle h, int n, int k, const double* A, int lda,
                                       double* C, int ldc, int k_tile)
{
    if (!h) return;
    if (n <= 0 || k <= 0) { record(h, HDBF_STATUS_SUCCESS); return; }
    const int tk = (k_tile <= 0 || k_tile >= k) ? k : k_tile;
    hdbf_status st = HDBF_STATUS_SUCCESS;
    for (int k0 = 0; k0 < k && st == HDBF_STATUS_SUCCESS; k0 += tk)
        st = syrk_lower(h, n, std::min(tk, k - k0), A + (long long)k0 * lda, lda, C, ldc);
    record(h, st);
}

void recursive_syrk_parallel_double(hdbf_handle h, double* A, int lda, double* C, int ldc, int n,
                                    int k, int nb)
{
    HDBF_ABI(h, rec_syrk_impl(h, A, lda, C, ldc, n, k, nb));
}

void batched_syrk_bottom_up_double(hdbf_handle h, StreamPool* pool, double* A, int lda,
                                   double* C, int ldc, int n, int k, int nb)
{
    (void)pool;
    HDBF_ABI(h, batched_syrk_impl(h, A, lda, C, ldc, n, k, nb));
}

void trsm_right_lower_transpose_double(hdbf_handle h, int rows, int cols, const double* A,
                                       int lda, double* B, int ldb)
{
    HDBF_ABI(h, trsm_rlt(h, rows, cols, A, lda, B, ldb));
}

void double_blocked_trsm_double(hdbf_handle h, double* A, int lda, double* B, int ldb, int n,
                                int m, int nb, int b)
{
    HDBF_ABI(h, dbtrsm_impl(h, A, lda, B, ldb, n, m, nb, b));
}

void recursive_trsm_double(hdbf_handle h, double* A, int lda, double* B, int ldb, int n, int m,
                           int nb)
{
    HDBF_ABI(h, rec_trsm_impl(h, A, lda, B, ldb, n, m, nb, false));
}

void gemm_nt_update_double(hdbf_handle h, int rows, int cols, int k, const double* A, int lda,
                           const double* B, int ldb, double* C, int ldc)
{
    HDBF_ABI(h, gemm_sub(h, false, false, rows, cols, k, A, lda, B, ldb, C, ldc));
}

void gemm_nt_update_m_tiled_double(hdbf_handle h, int rows, int cols, int k, const double* A,
                                   int lda, const double* B, int ldb, double* C, int ldc,
                                   int m_tile)
{
    HDBF_ABI(h, gemm_nt_rows(h, rows, cols, k, A, lda, B, ldb, C, ldc, m_tile, false));
}

}  // extern "C"
