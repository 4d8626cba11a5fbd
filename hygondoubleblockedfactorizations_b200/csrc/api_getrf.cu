// C ABI: LU drivers and the row-interchange launchers.
#include <algorithm>
#include <mutex>

#include "internal.h"
#include "getrf/blocked_getrf.h"
#include "getrf/blocked_getrf_npvt.h"
#include "getrf/double_blocked_getrf.h"
#include "getrf/double_blocked_getrf_npvt.h"
#include "getrf/getrf_pivot_kernels.h"

namespace hdbf {
namespace {

template <class T>
inline T* at(T* A, long long lda, int r, int c) { return A + (long long)c * lda + r; }

// The row-move scratch of a workspace, in the factorization's scalar type.
template <class T>
inline T* ws_temp(const GetrfWs& ws) { return reinterpret_cast<T*>(ws.temp); }

hdbf_status record(hdbf_context* ctx, hdbf_status st)
{
    if (ctx) ctx->last_status = st;
    return st;
}

bool bad_matrix(const void* A, int lda, int rows)
{
    return rows < 0 || (rows > 0 && (!A || lda < std::max(1, rows)));
}

__global__ void offset_pivots_kernel(int* p, int k, int delta)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < k) p[i] += delta;
}

// Compose the swaps ipiv[0..k) (1-based, minus `minus` gives rows local to
// A(row0:n, :)) and apply them to columns [c0, c0+nc) of rows row0..n.
template <class T>
hdbf_status permute_cols(hdbf_context* ctx, const GetrfWs& ws, T* A, long long lda, int n,
                         int row0, const int* ipiv, int k, int minus, int* info,
                         const int* col_begin, const int* col_count, int ranges)
{
    const int m = n - row0;
    if (k <= 0 || m <= 0) return HDBF_STATUS_SUCCESS;
    bool any = false;
    for (int r = 0; r < ranges; ++r) any = any || col_count[r] > 0;
    if (!any) return HDBF_STATUS_SUCCESS;
    HDBF_TRY(compose_swaps(ctx, ipiv, k, minus, m, ws.src, ws.tgt, ws.count, ws.gperm, info));
    const int max_moves = std::min(m, 2 * k);
    for (int r = 0; r < ranges; ++r)
        if (col_count[r] > 0)
            HDBF_TRY(apply_moves(ctx, at(A, lda, row0, col_begin[r]), lda, col_count[r], ws.src,
                                 ws.tgt, ws.count, max_moves, ws_temp<T>(ws), ws.temp_cols));
    return HDBF_STATUS_SUCCESS;
}

// L11^{-1} applied to B (rows x cols), direct or in trsm_block row blocks
// (src/getrf/getrf_pivot_internal.h:64-110).
template <class T>
hdbf_status trsm_llu_mode(hdbf_context* ctx, int rows, int cols, T* L, long long ldl,
                          T* B, long long ldb, bool iterative, int block)
{
    if (!iterative || block <= 0 || rows <= block) {
        StageScope sc(ctx, kStOuterTrsmDirect);
        return trsm_llu(ctx, rows, cols, L, ldl, B, ldb);
    }
    for (int r = 0; r < rows; r += block) {
        const int dr = std::min(block, rows - r);
        {
            StageScope sc(ctx, kStOuterTrsmBlock);
            HDBF_TRY(trsm_llu(ctx, dr, cols, at(L, ldl, r, r), ldl, B + r, ldb));
        }
        const int tr = rows - r - dr;
        if (tr > 0) {
            StageScope sc(ctx, kStOuterTrsmGemm);
            HDBF_TRY(gemm_sub(ctx, true, false, tr, cols, dr, at(L, ldl, r + dr, r), ldl, B + r,
                               ldb, B + r + dr, ldb));
        }
    }
    return HDBF_STATUS_SUCCESS;
}

// C -= L * U in row chunks (inner GEMM M-tiling,
// src/getrf/getrf_batched_pivot_internal.h:285-323).
template <class T>
hdbf_status gemm_nn_rows(hdbf_context* ctx, int rows, int cols, int k, const T* L,
                         long long ldl, const T* U, long long ldu, T* C, long long ldc,
                         int m_tile)
{
    const int tile = m_tile > 0 ? m_tile : std::max(rows, 1);
    for (int r = 0; r < rows; r += tile)
        HDBF_TRY(gemm_sub(ctx, true, false, std::min(tile, rows - r), cols, k, L + r, ldl, U,
                           ldu, C + r, ldc));
    return HDBF_STATUS_SUCCESS;
}

enum class PivotMode { Immediate, Batched, None };

// Launchers enqueue on ctx->stream; the look-ahead panel chain points it at
// the internal stream for the duration of a scope.
struct OnStream {
    hdbf_context* ctx;
    cudaStream_t saved;
    OnStream(hdbf_context* c, cudaStream_t s) : ctx(c), saved(c->stream) { c->stream = s; }
    ~OnStream() { ctx->stream = saved; }
};

struct NoSkinny {
    hdbf_context* ctx;
    explicit NoSkinny(hdbf_context* c) : ctx(c) { c->no_skinny = true; }
    ~NoSkinny() { ctx->no_skinny = false; }
};

// Double-blocked left-looking LU (src/getrf/double_blocked_getrf.cpp:125-191,
// src/getrf/getrf_batched_pivot_internal.h:445-624,
// src/getrf/double_blocked_getrf_npvt.cpp:93-144).
//
// Look-ahead (batched or no pivoting, hdbf_set_lookahead): the outer TRSM of
// block b+1 runs whole, then its outer GEMM (K = all previous columns) is
// enqueued on the caller's stream in column chunks of whole inner panels,
// each followed by an event; the inner-panel chain of block b+1 (panel, row
// interchanges, inner TRSM + GEMM) runs on the high-priority internal stream
// and waits only for the chunk it is about to touch, so panel factorizations
// overlap the rest of the outer GEMM.  The chain joins the caller's stream
// before the block's outer pivot batch.  Interchanges of a block's panels
// reach each later inner panel of the block as one composed permutation just
// before its inner update (instead of one permutation per panel), because
// the outer GEMM may still be writing those columns; the composition is kept
// running across the block's panels, and the data movement is the same.
template <class T>
hdbf_status getrf_db_impl(hdbf_context* ctx, T* A, int lda, int n, int outer_nb,
                          int inner_nb, bool iterative_outer, int trsm_block,
                          int inner_gemm_m_tile, int* ipiv, int* info, PivotMode mode,
                          const getrf_batched_pivot_workspace* user_ws)
{
    if (bad_matrix(A, lda, n)) return HDBF_STATUS_INVALID_VALUE;
    if (mode != PivotMode::None && n > 0 && !ipiv) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0) {
        if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
        return last_cuda(ctx);
    }
    GetrfWs ws;
    HDBF_TRY(getrf_workspace(ctx, ws_order<T>(n), &ws));
    if (mode == PivotMode::Batched && user_ws) {
        ws.src = user_ws->device_sources;
        ws.tgt = user_ws->device_targets;
        ws.temp = static_cast<float*>(user_ws->device_swap_buffer);
        ws.temp_cols = user_ws->column_tile;
    }
    if (outer_nb <= 0) outer_nb = n;
    if (inner_nb <= 0) inner_nb = outer_nb;
    inner_nb = std::min(inner_nb, outer_nb);
    const bool piv = mode != PivotMode::None;
    bool la = sizeof(T) == 4 && ctx->lookahead && mode != PivotMode::Immediate && n > outer_nb &&
              compose_running_fits(ctx, n, inner_nb);
    if (la && !ctx->la_stream) {
        // The stream and events are created outside any capture.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess ||
            cs != cudaStreamCaptureStatusNone || ensure_lookahead(ctx) != HDBF_STATUS_SUCCESS) {
            cudaGetLastError();
            la = false;
        }
    }
    const std::vector<long long> key = {
        10 + (int)mode + type_tag<T>(), (long long)A, lda, n, outer_nb, inner_nb, iterative_outer, trsm_block,
        inner_gemm_m_tile, (long long)ipiv, (long long)info, (long long)ws.src, (long long)ws.tgt,
        (long long)ws.temp, ws.temp_cols, la ? 1 : 0};
    return run_graph(ctx, key, [&]() -> hdbf_status {
    if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
    const cudaStream_t main_s = ctx->stream;
    int nchunks = 0;  // outer-update chunks of the current block (look-ahead)
    int chunk_w = 0;  // their width in columns (whole inner panels)

    // Inner panels of one outer block [outer, oend).
    auto block_chain = [&](int outer, int oend, bool forked) -> hdbf_status {
        int waited = 0;
        auto wait_chunk = [&](int col) {
            const int c = (col - outer) / chunk_w;
            while (waited <= c && waited < nchunks)
                cudaStreamWaitEvent(ctx->stream, ctx->la_ev[waited++], 0);
        };
        if (forked) wait_chunk(outer);
        for (int inner = outer; inner < oend; inner += inner_nb) {
            const int isz = std::min(inner_nb, oend - inner);
            const int next = inner + isz;
            {
                StageScope sc(ctx, kStPanel);
                HDBF_TRY(getrf_panel(ctx, n - inner, isz, at(A, lda, inner, inner), lda,
                                     piv ? ipiv + inner : nullptr, inner, info, inner, piv, ws));
            }
            if (mode == PivotMode::Immediate) {
                StageScope sc(ctx, kStPivotProp);
                const int cb[2] = {0, next};
                const int cc[2] = {inner, n - next};
                HDBF_TRY(permute_cols(ctx, ws, A, lda, n, inner, ipiv + inner, isz, inner, info,
                                      cb, cc, 2));
            } else if (mode == PivotMode::Batched) {
                StageScope sc(ctx, kStInnerPivot);
                const int cb[2] = {outer, next};
                const int cc[2] = {inner - outer, la ? 0 : oend - next};
                HDBF_TRY(permute_cols(ctx, ws, A, lda, n, inner, ipiv + inner, isz, inner, info,
                                      cb, cc, 2));
            }
            if (next < oend) {  // prepare_next_inner_panel
                const int nsz = std::min(inner_nb, oend - next);
                const int hist = next - outer;
                if (forked) wait_chunk(next);
                if (la && mode == PivotMode::Batched) {  // the block's interchanges so far
                    StageScope sc(ctx, kStInnerPivot);
                    HDBF_TRY(compose_running(ctx, ipiv + outer, inner - outer, hist, outer,
                                             n - outer, ws_perm(ctx), inner == outer, ws.src,
                                             ws.tgt, ws.count, info));
                    HDBF_TRY(apply_moves(ctx, at(A, lda, outer, next), lda, nsz, ws.src, ws.tgt,
                                         ws.count, std::min(n - outer, 2 * hist),
                                         ws_temp<T>(ws), ws.temp_cols));
                }
                {
                    StageScope sc(ctx, kStInnerTrsm);
                    HDBF_TRY(trsm_llu(ctx, hist, nsz, at(A, lda, outer, outer), lda,
                                      at(A, lda, outer, next), lda));
                }
                StageScope sc(ctx, kStInnerGemm);
                HDBF_TRY(gemm_nn_rows(ctx, n - next, nsz, hist, at(A, lda, next, outer), lda,
                                      at(A, lda, outer, next), lda, at(A, lda, next, next), lda,
                                      mode == PivotMode::Batched ? inner_gemm_m_tile : 0));
            }
        }
        return HDBF_STATUS_SUCCESS;
    };

    for (int outer = 0; outer < n; outer += outer_nb) {
        const int oend = outer + std::min(outer_nb, n - outer);
        if (nchunks > 0) {
            ctx->la_used = true;
            hdbf_status st;
            {
                OnStream on(ctx, ctx->la_stream);
                st = block_chain(outer, oend, true);
                cudaEventRecord(ctx->la_ev[kLaEvents - 1], ctx->la_stream);
            }
            cudaStreamWaitEvent(main_s, ctx->la_ev[kLaEvents - 1], 0);
            HDBF_TRY(st);
        } else {
            HDBF_TRY(block_chain(outer, oend, false));
        }
        nchunks = 0;
        if (mode == PivotMode::Batched) {  // outer pivot batch (:556-609)
            StageScope sc(ctx, kStOuterPivot);
            if (outer > 0) {
                const int cb[1] = {0};
                const int cc[1] = {outer};
                HDBF_TRY(permute_cols(ctx, ws, A, lda, n, outer, ipiv + outer, oend - outer, outer,
                                      info, cb, cc, 1));
            }
            if (oend < n) {
                const int cb[1] = {oend};
                const int cc[1] = {std::min(outer_nb, n - oend)};
                HDBF_TRY(permute_cols(ctx, ws, A, lda, n, 0, ipiv, oend, 0, info, cb, cc, 1));
            }
        }
        if (oend < n) {  // prepare_next_outer_panel
            const int next = oend;
            const int nsz = std::min(outer_nb, n - next);
            HDBF_TRY(trsm_llu_mode(ctx, next, nsz, A, lda, at(A, lda, 0, next), lda,
                                   iterative_outer, trsm_block));
            StageScope sc(ctx, kStOuterGemm);
            if (la) {
                const int panels = (nsz + inner_nb - 1) / inner_nb;
                const int group = (panels + kLaEvents - 2) / (kLaEvents - 1);
                chunk_w = group * inner_nb;
                NoSkinny ns(ctx);  // the panel chain may use the split-K scratch
                SplitPlan sp(ctx, n - next, nsz, next);  // chunks sum as the whole GEMM
                for (int c0 = 0; c0 < nsz; c0 += chunk_w) {
                    const int cw = std::min(chunk_w, nsz - c0);
                    HDBF_TRY(gemm_sub(ctx, true, false, n - next, cw, next, at(A, lda, next, 0),
                                       lda, at(A, lda, 0, next + c0), lda,
                                       at(A, lda, next, next + c0), lda));
                    cudaEventRecord(ctx->la_ev[nchunks++], main_s);
                }
            } else {
                HDBF_TRY(gemm_sub(ctx, true, false, n - next, nsz, next, at(A, lda, next, 0), lda,
                                   at(A, lda, 0, next), lda, at(A, lda, next, next), lda));
            }
        }
    }
    return last_cuda(ctx);
    });
}

// Blocked right-looking LU (src/getrf/blocked_getrf.cpp:15-71).
template <class T>
hdbf_status getrf_rl_impl(hdbf_context* ctx, T* A, int lda, int n, int nb, int* ipiv,
                          int* info, bool piv)
{
    if (bad_matrix(A, lda, n)) return HDBF_STATUS_INVALID_VALUE;
    if (piv && n > 0 && !ipiv) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0) {
        if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
        return last_cuda(ctx);
    }
    GetrfWs ws;
    HDBF_TRY(getrf_workspace(ctx, ws_order<T>(n), &ws));
    if (nb <= 0) nb = n;
    const std::vector<long long> key = {20 + (int)piv + type_tag<T>(), (long long)A, lda, n, nb, (long long)ipiv,
                                        (long long)info};
    return run_graph(ctx, key, [&]() -> hdbf_status {
    if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
    for (int p = 0; p < n; p += nb) {
        const int psz = std::min(nb, n - p);
        const int next = p + psz;
        const int tr = n - next;
        HDBF_TRY(getrf_panel(ctx, n - p, psz, at(A, lda, p, p), lda, piv ? ipiv + p : nullptr, p,
                             info, p, piv, ws));
        if (piv) {
            const int cb[2] = {0, next};
            const int cc[2] = {p, tr};
            HDBF_TRY(permute_cols(ctx, ws, A, lda, n, p, ipiv + p, psz, p, info, cb, cc, 2));
        }
        if (tr > 0) {
            HDBF_TRY(trsm_llu(ctx, psz, tr, at(A, lda, p, p), lda, at(A, lda, p, next), lda));
            HDBF_TRY(gemm_sub(ctx, true, false, tr, tr, psz, at(A, lda, next, p), lda,
                               at(A, lda, p, next), lda, at(A, lda, next, next), lda));
        }
    }
    return last_cuda(ctx);
    });
}

bool batched_ws_valid(const getrf_batched_pivot_workspace* w, int n)
{
    // src/getrf/getrf_batched_pivot_internal.h:43-57
    return w && w->device_sources && w->device_targets && w->device_swap_buffer &&
           w->host_pivots && w->host_permutation && w->host_sources && w->host_targets &&
           w->capacity >= n && w->column_tile > 0;
}

// Context used by the handle-less kernel launchers.
hdbf_context* launcher_context(cudaStream_t stream)
{
    static std::mutex mu;
    static hdbf_context* ctx = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!ctx) {
        if (hdbf_create(&ctx) != HDBF_STATUS_SUCCESS) return nullptr;
    }
    ctx->stream = stream;
    return ctx;
}

}  // namespace
}  // namespace hdbf

using namespace hdbf;

extern "C" {

void double_blocked_getrf(hdbf_handle h, float* A, int lda, int n, int outer_nb, int inner_nb,
                          getrf_outer_trsm_mode outer_trsm_mode, int trsm_block, int* ipiv,
                          int* info)
{
    if (!h) return;
    record(h, getrf_db_impl(h, A, lda, n, outer_nb, inner_nb,
                            outer_trsm_mode == getrf_outer_trsm_iterative, trsm_block, 0, ipiv,
                            info, PivotMode::Immediate, nullptr));
}

void double_blocked_getrf_batched_pivot(hdbf_handle h, float* A, int lda, int n, int outer_nb,
                                        int inner_nb, getrf_outer_trsm_mode outer_trsm_mode,
                                        int trsm_block, int inner_gemm_m_tile, int* ipiv,
                                        int* info, getrf_batched_pivot_workspace* workspace)
{
    if (!h) return;
    if (!batched_ws_valid(workspace, n)) {
        // double_blocked_getrf.cpp:263-267: info = -1 via a 0xff memset
        if (info) cudaMemsetAsync(info, 0xff, sizeof(int), h->stream);
        record(h, HDBF_STATUS_INVALID_VALUE);
        return;
    }
    record(h, getrf_db_impl(h, A, lda, n, outer_nb, inner_nb,
                            outer_trsm_mode == getrf_outer_trsm_iterative, trsm_block,
                            inner_gemm_m_tile, ipiv, info, PivotMode::Batched, workspace));
}

void double_blocked_getrf_npvt(hdbf_handle h, float* A, int lda, int n, int nb, int b, int* info)
{
    if (!h) return;
    record(h, getrf_db_impl(h, A, lda, n, nb, b, false, 0, 0, nullptr, info, PivotMode::None,
                            nullptr));
}

void blocked_right_looking_getrf(hdbf_handle h, float* A, int lda, int n, int nb, int* ipiv,
                                 int* info)
{
    if (!h) return;
    record(h, getrf_rl_impl(h, A, lda, n, nb, ipiv, info, true));
}

void blocked_right_looking_getrf_npvt(hdbf_handle h, float* A, int lda, int n, int nb, int* info)
{
    if (!h) return;
    record(h, getrf_rl_impl(h, A, lda, n, nb, nullptr, info, false));
}

void launch_apply_getrf_panel_pivots(float* A, int lda, int n, int panel, int panel_size,
                                     int* pivots, cudaStream_t stream)
{
    if (!A || !pivots || panel_size <= 0 || n <= 0) return;
    hdbf_context* ctx = launcher_context(stream);
    if (!ctx) return;
    GetrfWs ws;
    if (getrf_workspace(ctx, n, &ws) != HDBF_STATUS_SUCCESS) return;
    const int next = panel + panel_size;
    const int cb[2] = {0, next};
    const int cc[2] = {panel, n - next};
    if (permute_cols(ctx, ws, A, lda, n, panel, pivots, panel_size, 0, nullptr, cb, cc, 2) !=
        HDBF_STATUS_SUCCESS)
        return;
    offset_pivots_kernel<<<(panel_size + 255) / 256, 256, 0, stream>>>(pivots, panel_size, panel);
}

void launch_apply_getrf_permutation(float* A, int lda, int column_count, const int* sources,
                                    const int* targets, int move_count, float* temporary,
                                    int column_tile, cudaStream_t stream)
{
    if (!A || column_count <= 0 || move_count <= 0 || column_tile <= 0) return;
    hdbf_context* ctx = launcher_context(stream);
    if (!ctx) return;
    // The move count is a host value here; stage it into the device word.
    int* cnt = ctx->dev_small + kSmallMoveCount + 1;
    cudaMemcpyAsync(cnt, &move_count, sizeof(int), cudaMemcpyHostToDevice, stream);
    apply_moves(ctx, A, lda, column_count, sources, targets, cnt, move_count, temporary,
                column_tile);
}

// ------------------------------------------------------------ FP64 twins
// The reference's `_double` LU entry points: the same drivers instantiated
// for double on this library's FP64 kernels (fp64.cu).

void double_blocked_getrf_double(hdbf_handle h, double* A, int lda, int n, int outer_nb,
                                 int inner_nb, getrf_outer_trsm_mode outer_trsm_mode,
                                 int trsm_block, int* ipiv, int* info)
{
    if (!h) return;
    record(h, getrf_db_impl(h, A, lda, n, outer_nb, inner_nb,
                            outer_trsm_mode == getrf_outer_trsm_iterative, trsm_block, 0, ipiv,
                            info, PivotMode::Immediate, nullptr));
}

void double_blocked_getrf_double_batched_pivot(hdbf_handle h, double* A, int lda, int n,
                                               int outer_nb, int inner_nb,
                                               getrf_outer_trsm_mode outer_trsm_mode,
                                               int trsm_block, int inner_gemm_m_tile, int* ipiv,
                                               int* info, getrf_batched_pivot_workspace* workspace)
{
    if (!h) return;
    if (!batched_ws_valid(workspace, n)) {
        if (info) cudaMemsetAsync(info, 0xff, sizeof(int), h->stream);
        record(h, HDBF_STATUS_INVALID_VALUE);
        return;
    }
    record(h, getrf_db_impl(h, A, lda, n, outer_nb, inner_nb,
                            outer_trsm_mode == getrf_outer_trsm_iterative, trsm_block,
                            inner_gemm_m_tile, ipiv, info, PivotMode::Batched, workspace));
}

void double_blocked_getrf_npvt_double(hdbf_handle h, double* A, int lda, int n, int nb, int b,
                                      int* info)
{
    if (!h) return;
    record(h, getrf_db_impl(h, A, lda, n, nb, b, false, 0, 0, nullptr, info, PivotMode::None,
                            nullptr));
}

void blocked_right_looking_getrf_double(hdbf_handle h, double* A, int lda, int n, int nb,
                                        int* ipiv, int* info)
{
    if (!h) return;
    record(h, getrf_rl_impl(h, A, lda, n, nb, ipiv, info, true));
}

void blocked_right_looking_getrf_npvt_double(hdbf_handle h, double* A, int lda, int n, int nb,
                                             int* info)
{
    if (!h) return;
    record(h, getrf_rl_impl(h, A, lda, n, nb, nullptr, info, false));
}

void launch_apply_getrf_panel_pivots_double(double* A, int lda, int n, int panel,
                                            int panel_size, int* pivots, cudaStream_t stream)
{
    if (!A || !pivots || panel_size <= 0 || n <= 0) return;
    hdbf_context* ctx = launcher_context(stream);
    if (!ctx) return;
    GetrfWs ws;
    if (getrf_workspace(ctx, ws_order<double>(n), &ws) != HDBF_STATUS_SUCCESS) return;
    const int next = panel + panel_size;
    const int cb[2] = {0, next};
    const int cc[2] = {panel, n - next};
    if (permute_cols(ctx, ws, A, lda, n, panel, pivots, panel_size, 0, nullptr, cb, cc, 2) !=
        HDBF_STATUS_SUCCESS)
        return;
    offset_pivots_kernel<<<(panel_size + 255) / 256, 256, 0, stream>>>(pivots, panel_size, panel);
}

void launch_apply_getrf_permutation_double(double* A, int lda, int column_count,
                                           const int* sources, const int* targets,
                                           int move_count, double* temporary, int column_tile,
                                           cudaStream_t stream)
{
    if (!A || column_count <= 0 || move_count <= 0 || column_tile <= 0) return;
    hdbf_context* ctx = launcher_context(stream);
    if (!ctx) return;
    int* cnt = ctx->dev_small + kSmallMoveCount + 1;
    cudaMemcpyAsync(cnt, &move_count, sizeof(int), cudaMemcpyHostToDevice, stream);
    apply_moves(ctx, A, lda, column_count, sources, targets, cnt, move_count, temporary,
                column_tile);
}

}  // extern "C"
