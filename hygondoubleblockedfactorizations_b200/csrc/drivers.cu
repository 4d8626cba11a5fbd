// Host-side building blocks: recursive diagonal Cholesky, recursive TRSMs,
// SYRK, recursive GETRF panel.  Everything is enqueued on ctx->stream; no
// host synchronisation.
#include <algorithm>

#include "internal.h"

namespace hdbf {

namespace {
constexpr int kDiagLeaf = 64;   // potf2_small / trsm_*_small leaf order
constexpr int kClusterLeaf = 32;  // widest block of the cluster panel kernel

// Split point for a recursion on `n` columns with `leaf`-aligned halves.
inline int split_at(int n, int leaf)
{
    int h = (n / 2 + leaf - 1) / leaf * leaf;
    if (h <= 0 || h >= n) h = std::max(1, n - leaf);
    return h;
}
}  // namespace

hdbf_status potrf_diag(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                       int info_base)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    if (n <= kDiagLeaf) return potf2_small(ctx, n, A, lda, info, info_base);
    if (n <= potrf_block_max_n()) return potrf_block(ctx, n, A, lda, info, info_base, nullptr, 0);
    const int n1 = split_at(n, kDiagLeaf);
    const int n2 = n - n1;
    float* A21 = A + n1;
    float* A22 = A + (long long)n1 * lda + n1;
    HDBF_TRY(potrf_diag(ctx, n1, A, lda, info, info_base));
    HDBF_TRY(trsm_rlt(ctx, n2, n1, A, lda, A21, lda));
    HDBF_TRY(syrk_lower(ctx, n2, n1, A21, lda, A22, lda));
    return potrf_diag(ctx, n2, A22, lda, info, info_base + n1);
}

namespace {
// Recursive right/lower/transposed solve with precomputed 64x64 block inverses
// (inv holds the blocks of L starting at block `blk`).
hdbf_status trsm_rlt_rec(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                         float* B, long long ldb, const float* inv)
{
    if (cols <= kDiagLeaf) return rlt_apply(ctx, rows, cols, inv, B, ldb);
    if (cols <= llu_block_max_rows()) return rlt_block(ctx, rows, cols, L, ldl, inv, B, ldb);
    const int c1 = split_at(cols, kDiagLeaf);
    const int c2 = cols - c1;
    HDBF_TRY(trsm_rlt_rec(ctx, rows, c1, L, ldl, B, ldb, inv));
    // B2 -= X1 * L21^T, L21 = L(c1:cols, 0:c1)
    HDBF_TRY(sgemm_sub(ctx, false, false, rows, c2, c1, B, ldb, L + c1, ldl,
                       B + (long long)c1 * ldb, ldb));
    return trsm_rlt_rec(ctx, rows, c2, L + (long long)c1 * ldl + c1, ldl,
                        B + (long long)c1 * ldb, ldb, inv + (long long)(c1 / kDiagLeaf) * 4096);
}

hdbf_status trsm_llu_rec(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                         float* B, long long ldb, const float* inv)
{
    if (rows <= kDiagLeaf) return llu_apply(ctx, rows, cols, inv, B, ldb);
    if (rows <= llu_block_max_rows()) return llu_block(ctx, rows, cols, L, ldl, inv, B, ldb);
    const int r1 = split_at(rows, kDiagLeaf);
    const int r2 = rows - r1;
    HDBF_TRY(trsm_llu_rec(ctx, r1, cols, L, ldl, B, ldb, inv));
    // B2 -= L21 * X1
    HDBF_TRY(sgemm_sub(ctx, true, false, r2, cols, r1, L + r1, ldl, B, ldb, B + r1, ldb));
    return trsm_llu_rec(ctx, r2, cols, L + (long long)r1 * ldl + r1, ldl, B + r1, ldb,
                        inv + (long long)(r1 / kDiagLeaf) * 4096);
}
}  // namespace

// B(rows x cols) <- B * L^{-T}: invert the 64x64 diagonal blocks of L once,
// then recurse on column halves with GEMM updates; leaves are small GEMMs
// with the inverted blocks (no serial dependency chains).
hdbf_status trsm_rlt(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                     float* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    HDBF_TRY(ensure_ws(ctx, cols));
    float* inv = ws_inv(ctx);
    HDBF_TRY(tri_inv64(ctx, cols, L, ldl, false, inv));
    return trsm_rlt_rec(ctx, rows, cols, L, ldl, B, ldb, inv);
}

// B(rows x cols) <- L^{-1} B, L unit lower, same scheme on row halves.
hdbf_status trsm_llu(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                     float* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    HDBF_TRY(ensure_ws(ctx, rows));
    float* inv = ws_inv(ctx);
    HDBF_TRY(tri_inv64(ctx, rows, L, ldl, true, inv));
    return trsm_llu_rec(ctx, rows, cols, L, ldl, B, ldb, inv);
}

hdbf_status syrk_lower(hdbf_context* ctx, int n, int k, const float* A, long long lda,
                       float* C, long long ldc)
{
    return sgemm_sub(ctx, false, true, n, n, k, A, lda, A, lda, C, ldc);
}

hdbf_status getrf_workspace(hdbf_context* ctx, int n, GetrfWs* ws)
{
    HDBF_TRY(ensure_ws(ctx, n));
    ws->src = ws_src(ctx);
    ws->tgt = ws_tgt(ctx);
    ws->gperm = ws_gperm(ctx);
    ws->temp = ws_temp(ctx);
    ws->temp_cols = 64;
    ws->count = ctx->dev_small + kSmallMoveCount;
    return HDBF_STATUS_SUCCESS;
}

// Recursive (Toledo/Gustavson) LU of an m x w panel.  Leaves are column
// blocks of the handle's panel-leaf width (default 128; 32 when the cluster
// kernel is forced) and go to the cluster kernel when they fit in one cluster
// (w <= 32), otherwise to the grid-wide kernel.  ipiv receives (local row + 1
// + ipiv_add) for the panel's w columns.
hdbf_status getrf_panel(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                        int ipiv_add, int* info, int info_base, bool pivot, const GetrfWs& ws)
{
    if (m <= 0 || w <= 0) return HDBF_STATUS_SUCCESS;
    const int leaf = ctx->panel_mode == 2 ? kClusterLeaf : ctx->panel_leaf;
    if (w <= leaf) {
        if (ctx->panel_mode != 1 && w <= kClusterLeaf) {
            const hdbf_status st =
                getf2_cluster(ctx, m, w, A, lda, ipiv, ipiv_add, info, info_base, pivot);
            if (st != HDBF_STATUS_NOT_SUPPORTED) return st;
        }
        return getf2_coop(ctx, m, w, A, lda, ipiv, ipiv_add, info, info_base, pivot);
    }
    const int w1 = split_at(w, leaf);
    const int w2 = w - w1;
    HDBF_TRY(getrf_panel(ctx, m, w1, A, lda, ipiv, ipiv_add, info, info_base, pivot, ws));
    float* A12 = A + (long long)w1 * lda;
    if (pivot) {
        HDBF_TRY(compose_swaps(ctx, ipiv, w1, ipiv_add, m, ws.src, ws.tgt, ws.count, ws.gperm,
                               info));
        HDBF_TRY(apply_moves(ctx, A12, lda, w2, ws.src, ws.tgt, ws.count,
                             std::min(m, 2 * w1), ws.temp, ws.temp_cols));
    }
    HDBF_TRY(trsm_llu(ctx, w1, w2, A, lda, A12, lda));
    HDBF_TRY(sgemm_sub(ctx, true, false, m - w1, w2, w1, A + w1, lda, A12, lda, A12 + w1, lda));
    HDBF_TRY(getrf_panel(ctx, m - w1, w2, A12 + w1, lda, pivot ? ipiv + w1 : nullptr,
                         ipiv_add + w1, info, info_base + w1, pivot, ws));
    if (pivot) {
        HDBF_TRY(compose_swaps(ctx, ipiv + w1, w2, ipiv_add + w1, m - w1, ws.src, ws.tgt,
                               ws.count, ws.gperm, info));
        HDBF_TRY(apply_moves(ctx, A + w1, lda, w1, ws.src, ws.tgt, ws.count,
                             std::min(m - w1, 2 * w2), ws.temp, ws.temp_cols));
    }
    return HDBF_STATUS_SUCCESS;
}

}  // namespace hdbf
