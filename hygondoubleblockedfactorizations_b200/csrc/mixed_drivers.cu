// Mixed-precision factorizations: FP32 panels, tensor-core trailing updates.
//
// Cholesky and LU run right-looking with block b: the diagonal block / tall
// panel is factored in FP32 by the same kernels as the FP32 path (potf2 +
// inverted-block TRSM; cooperative pivoted panel + device-composed row swaps),
// the off-diagonal panel(s) are rounded once into K-major 16-bit shadows, and
// the O(n^3) trailing update A22 -= L21 L21^T (SYRK, lower) or A22 -= L21 U12
// runs on tcgen05 with FP32 accumulation straight into the FP32 matrix.  In
// the split modes each operand is carried as hi + lo (lo = round(x - hi)) and
// the update uses hi*hi + hi*lo + lo*hi.
//
// Reference: the mixed recursive Cholesky (src/potrf/recursive_potrf.cpp:
// 241-388) rounds C to FP16 in every GEMM (src/gemm/mixed_gemm.cpp:53-89);
// here C never leaves FP32.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"
#include "hdbf/mixed.h"
#include "kernels/add_damping.h"
#include "potrf/recursive_potrf.h"
#include "syrk/batched_syrk.h"
#include "trsm/recursive_trsm.h"

namespace hdbf {

size_t mixed_base_bytes(int n, int b);
size_t mixed_slots_offset(int n, int b);

namespace {

inline long long pad8(long long x) { return (x + 7) / 8 * 8; }
inline float* at(float* A, long long lda, int r, int c) { return A + (long long)c * lda + r; }

struct PrecInfo {
    int fmt;
    bool split;
};

PrecInfo prec_info(int prec)
{
    switch (prec) {
    case HDBF_PREC_BF16: return {kFmtBF16, false};
    case HDBF_PREC_FP16: return {kFmtF16, false};
    case HDBF_PREC_BF16X3: return {kFmtBF16, true};
    case HDBF_PREC_FP16X3: return {kFmtF16, true};
    default: return {-1, false};
    }
}

// C -= scale * (A B^T) with optional hi/lo split operands.
// sa / sb (optional): device max slots of per-panel scaled operands.
hdbf_status tc_update(hdbf_context* ctx, const PrecInfo& pi, int M, int N, int K, const void* ah,
                      const void* al, long long lda, const void* bh, const void* bl, long long ldb,
                      float* C, long long ldc, float scale, bool lower,
                      const unsigned* sa = nullptr, const unsigned* sb = nullptr)
{
    TcOperand a, b;
    a.base = ah;
    a.ld = lda;
    b.base = bh;
    b.ld = ldb;
    if (!pi.split) return tc_gemm_sub(ctx, pi.fmt, M, N, K, a, b, C, ldc, scale, lower, sa, sb);
    TcOperand alo = a, blo = b;
    alo.base = al;
    blo.base = bl;
    return tc_gemm_sub_split(ctx, pi.fmt, M, N, K, a, alo, b, blo, C, ldc, scale, lower, sa, sb);
}

__global__ void absmax_kernel(const float* A, long long lda, int rows, int cols, int diag_only,
                              unsigned int* out)
{
    float v = 0.f;
    if (diag_only) {
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < rows;
             i += (long long)gridDim.x * blockDim.x)
            v = fmaxf(v, fabsf(A[i * lda + i]));
    } else {
        const long long total = (long long)rows * cols;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
             i += (long long)gridDim.x * blockDim.x)
            v = fmaxf(v, fabsf(A[(i / rows) * lda + i % rows]));
    }
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(v));
}

__global__ void set_identity_kernel(float* W, long long ldw, int n)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const long long c = blockIdx.y;
    if (r < n) W[c * ldw + r] = (r == c) ? 1.f : 0.f;
}

hdbf_status set_identity(hdbf_context* ctx, float* W, long long ldw, int n)
{
    dim3 g((n + 255) / 256, n);
    set_identity_kernel<<<g, 256, 0, ctx->stream>>>(W, ldw, n);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status zero_block(hdbf_context* ctx, float* A, long long lda, int rows, int cols)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    if (cudaMemset2DAsync(A, (size_t)lda * sizeof(float), 0, (size_t)rows * sizeof(float), cols,
                          ctx->stream) != cudaSuccess)
        return last_cuda(ctx);
    return HDBF_STATUS_SUCCESS;
}

// Panel TRSM of the mixed factorizations.  BF16 and FP16 modes: one
// tensor-core GEMM with the FP32 inverse block, BF16 operands (FP32 range, so
// the inverse needs no scaling); one product in BF16 mode, hi + lo split
// (three products, ~16 significant bits) in FP16 mode.  The split modes keep
// the FP32 TRSM: their factors must be accurate to ~2^-22, which 16-bit
// operands of an unscaled inverse cannot give.
bool trsm_on_tc(const PrecInfo& pi) { return !pi.split; }
PrecInfo trsm_prec(const PrecInfo& pi) { return {kFmtBF16, pi.fmt == kFmtF16}; }

// Inverse-block scratch inside the arena.
struct WBlock {
    float* W;
    long long ldw;
    void* wh;
    void* wl;
    long long ldws;
};
WBlock w_block(char* arena, int n, int b)
{
    WBlock w;
    char* p = arena + mixed_base_bytes(n, b);
    w.W = reinterpret_cast<float*>(p);
    w.ldw = pad8(b);
    p += align_up((size_t)b * pad8(b) * 4, 256);
    w.wh = p;
    p += align_up((size_t)b * pad8(b) * 2, 256);
    w.wl = p;
    w.ldws = pad8(b);
    return w;
}

}  // namespace

// max |A| (diag_only: max |A(i,i)|); synchronises the stream.
hdbf_status absmax_host(hdbf_context* ctx, const float* A, long long lda, int rows, int cols,
                        bool diag_only, float* out)
{
    unsigned int* d = reinterpret_cast<unsigned int*>(ctx->dev_small + kSmallScratch);
    cudaMemsetAsync(d, 0, sizeof(unsigned int), ctx->stream);
    absmax_kernel<<<1184, 256, 0, ctx->stream>>>(A, lda, rows, cols, diag_only ? 1 : 0, d);
    ctx->launches++;
    unsigned int bits = 0;
    if (cudaMemcpyAsync(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    float f;
    memcpy(&f, &bits, sizeof(f));
    *out = f;
    return HDBF_STATUS_SUCCESS;
}

// Arena: four n x pad8(b) 16-bit shadows (hi/lo of two operands; the
// panel-TRSM GEMM uses the lo halves as scratch in every mode), then the
// FP32 inverse block W (b x pad8(b)) and its hi/lo shadows.
size_t mixed_base_bytes(int n, int b) { return align_up((size_t)4 * n * pad8(b) * 2, 256); }
// After W: one max slot (FP32 bits, see panel_scale_exp) per panel for the
// per-panel scales of the FP16 shadows.
size_t mixed_slots_offset(int n, int b)
{
    const size_t w = align_up((size_t)b * pad8(b) * 4, 256) + 2 * align_up((size_t)b * pad8(b) * 2, 256);
    return mixed_base_bytes(n, b) + w;
}
// Slot region: per-panel scale slots, per-panel fallback flags, then the
// fallback counter (each panels + 2 words); after it the FP32 copy of the
// original matrix (n x n) the Cholesky panel fallback recomputes from.
size_t mixed_slot_words(int n, int b) { return (size_t)n / b + 2; }
size_t mixed_backup_offset(int n, int b)
{
    return mixed_slots_offset(n, b) + align_up(3 * mixed_slot_words(n, b) * sizeof(unsigned), 256);
}
size_t mixed_shadow_bytes(int n, int b, bool split)
{
    (void)split;
    return mixed_backup_offset(n, b) + align_up((size_t)n * n * sizeof(float), 256) + 1024;
}

namespace {

// dst(r, c) = src(r, c) for the lower trapezoid r >= c of a rows x cols block
// column, when *run_if != 0 (the panel fallback's restore of the originals).
__global__ void restore_lower_kernel(int rows, int cols, const float* src, long long lds,
                                     float* dst, long long ldd, const int* run_if)
{
    if (*run_if == 0) return;
    const long long total = (long long)rows * cols;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i / rows), r = (int)(i % rows);
        if (r >= c) dst[(long long)c * ldd + r] = src[(long long)c * lds + r];
    }
}

// A panel whose first attempt failed (*flag != 0): count it; when the FP32
// retry failed too, its info stands (the retry wrote it).
__global__ void count_fallback_kernel(const int* flag, unsigned* counter)
{
    if (*flag != 0) atomicAdd(counter, 1u);
}

// First panel: nothing precedes it to recompute, so its failure is final.
__global__ void promote_info_kernel(const int* flag, int* info)
{
    if (*flag != 0 && info) atomicCAS(info, 0, *flag);
}

}  // namespace

// Panel fallback of the mixed Cholesky: if the diagonal block of panel k
// (rows k.., psz columns) failed after the low-precision trailing updates
// (*flag != 0, set by the first attempt), the panel's block column is
// rebuilt in FP32 from the original matrix A0 -- A(k:n, k:k+psz) =
// A0(k:n, k:k+psz) - L(k:n, 0:k) L(k:k+psz, 0:k)^T with the FP32 GEMM -- and
// its diagonal block factored again, writing `info` only if that fails too.
// Every launch is conditional on *flag (RunIf), so the graph of the
// factorization does the extra work only for panels that need it.
hdbf_status potrf_panel_fallback(hdbf_context* ctx, float* A, long long lda, const float* A0,
                                 long long ld0, int n, int k, int psz, const int* flag,
                                 int* info, float* W, long long ldw, unsigned* counter)
{
    if (k == 0) {
        promote_info_kernel<<<1, 1, 0, ctx->stream>>>(flag, info);
        ctx->launches++;
        return last_cuda(ctx);
    }
    const int rows = n - k;
    RunIf ri(ctx, flag);
    const long long total = (long long)rows * psz;
    const int g = (int)std::min<long long>((total + 255) / 256, 8LL * ctx->sm_count);
    restore_lower_kernel<<<g, 256, 0, ctx->stream>>>(rows, psz, A0 + (long long)k * ld0 + k, ld0,
                                                       at(A, lda, k, k), lda, flag);
    ctx->launches++;
    HDBF_TRY(sgemm_sub(ctx, false, true, psz, psz, k, at(A, lda, k, 0), lda, at(A, lda, k, 0), lda,
                       at(A, lda, k, k), lda));
    if (rows > psz)
        HDBF_TRY(sgemm_sub(ctx, false, false, rows - psz, psz, k, at(A, lda, k + psz, 0), lda,
                           at(A, lda, k, 0), lda, at(A, lda, k + psz, k), lda));
    HDBF_TRY(potrf_block(ctx, psz, at(A, lda, k, k), lda, info, k, W, ldw));
    count_fallback_kernel<<<1, 1, 0, ctx->stream>>>(flag, counter);
    ctx->launches++;
    return last_cuda(ctx);
}

// Right-looking mixed Cholesky (lower) with block b; shadows in `arena`.
// BF16 (one product, no per-panel scale) pairs the panels: the first panel of
// a pair updates only the second panel's block column (K = b), and the
// trailing matrix takes both panels at once (K = 2b) from one shadow that
// holds the pair's columns side by side -- half the passes over the FP32
// trailing matrix, whose read-modify-write bounds the tensor-core update at
// K = b.  The other modes update after every panel.
hdbf_status potrf_mixed_body(hdbf_context* ctx, int prec, float* A, long long lda, int n, int b,
                             int* info, char* arena)
{
    const PrecInfo pi = prec_info(prec);
    if (pi.fmt < 0) return HDBF_STATUS_INVALID_VALUE;
    const bool pair = pi.fmt == kFmtBF16 && !pi.split && b % 8 == 0 && b < n;
    // pair: shadow and TRSM scratch of n x pad8(2b) each, inside the four
    // n x pad8(b) arrays of the arena
    const long long lds = pair ? pad8(2 * b) : pad8(b);
    const size_t one = (size_t)n * lds * 2;
    char* hi = arena;
    char* lo = pi.split ? arena + one : nullptr;
    char* scratch_hi = pair ? arena + one : hi;
    char* scratch_lo = pair ? nullptr : arena + one;
    // FP16 shadows carry a per-panel power-of-two scale (FP16's range is
    // narrow); BF16 has FP32's exponent range and needs none.
    unsigned* slots = reinterpret_cast<unsigned*>(arena + mixed_slots_offset(n, b));
    const size_t words = mixed_slot_words(n, b);
    int* fail_flags = reinterpret_cast<int*>(slots + words);
    unsigned* fallbacks = slots + 2 * words;
    const bool scaled = pi.fmt == kFmtF16;
    const PrecInfo tp = trsm_prec(pi);
    const WBlock wb = w_block(arena, n, b);
    // The panel fallback (BF16 / FP16 modes) rebuilds a failed panel from a
    // copy of the original matrix.
    float* A0 = trsm_on_tc(pi) ? reinterpret_cast<float*>(arena + mixed_backup_offset(n, b))
                               : nullptr;
    if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
    cudaMemsetAsync(fallbacks, 0, sizeof(unsigned), ctx->stream);
    if (A0)
        cudaMemcpy2DAsync(A0, (size_t)n * sizeof(float), A, (size_t)lda * sizeof(float),
                          (size_t)n * sizeof(float), n, cudaMemcpyDeviceToDevice, ctx->stream);
    for (int k = 0; k < n; k += b) {
        unsigned* slot = scaled ? slots + k / b : nullptr;
        const int psz = std::min(b, n - k);
        const int tr = n - k - psz;
        float* Akk = at(A, lda, k, k);
        const bool inv_tc = trsm_on_tc(pi) && tr > 0 && psz <= potrf_block_max_n();
        const bool second = pair && ((k / b) & 1);  // second panel of a pair
        const int k0 = second ? k - b : k;            // the pair's first column
        if (inv_tc) {
            int* flag = fail_flags + k / b;
            cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream);
            HDBF_TRY(potrf_block(ctx, psz, Akk, lda, flag, k, wb.W, wb.ldw));
            HDBF_TRY(potrf_panel_fallback(ctx, A, lda, A0, n, n, k, psz, flag, info, wb.W, wb.ldw,
                                          fallbacks));
        } else {
            HDBF_TRY(potrf_diag(ctx, psz, Akk, lda, info, k));
        }
        if (tr <= 0) continue;
        float* A21 = at(A, lda, k + psz, k);
        float* C22 = at(A, lda, k + psz, k + psz);
        // this panel's rows k + psz .. n in the shadow: pair mode keeps the
        // pair's panels side by side, rows counted from the pair's first column
        char* sh = pair ? hi + ((size_t)(k + psz - k0) * lds + (k - k0)) * 2 : hi;
        if (!inv_tc) {
            HDBF_TRY(trsm_rlt(ctx, tr, psz, Akk, lda, A21, lda));
        } else {
            // L21 = A21 L11^{-T} as one tensor-core GEMM with W = L11^{-1}
            // from the diagonal-block kernel; A21 is rounded into the scratch
            // and overwritten with the product (B operand W: A21 W^T).
            HDBF_TRY(convert_transpose16(ctx, tp.fmt, psz, psz, wb.W, wb.ldw, wb.wh,
                                         tp.split ? wb.wl : nullptr, wb.ldws, 1.f));
            HDBF_TRY(convert_transpose16(ctx, tp.fmt, tr, psz, A21, lda, scratch_hi,
                                         tp.split ? scratch_lo : nullptr, lds, 1.f));
            HDBF_TRY(zero_block(ctx, A21, lda, tr, psz));
            HDBF_TRY(tc_update(ctx, tp, tr, psz, psz, scratch_hi, scratch_lo, lds, wb.wh, wb.wl,
                               wb.ldws, A21, lda, -1.f, false));
        }
        if (slot) HDBF_TRY(panel_absmax(ctx, A21, lda, tr, psz, slot));
        HDBF_TRY(convert_transpose16(ctx, pi.fmt, tr, psz, A21, lda, sh, pi.split ? lo : nullptr,
                                     lds, 1.f, slot));
        if (!pair) {
            HDBF_TRY(tc_update(ctx, pi, tr, tr, psz, hi, lo, lds, hi, lo, lds, C22, lda, 1.f, true,
                               slot, slot));
        } else if (!second) {
            // the pair's second panel only (its block column, lower on top)
            const int nb2 = std::min(b, tr);
            HDBF_TRY(tc_update(ctx, pi, tr, nb2, psz, sh, nullptr, lds, sh, nullptr, lds, C22,
                               lda, 1.f, true, nullptr, nullptr));
        } else {
            // the trailing matrix: both panels of the pair, K = b + psz
            char* pr = hi + (size_t)(k + psz - k0) * lds * 2;
            HDBF_TRY(tc_update(ctx, pi, tr, tr, b + psz, pr, nullptr, lds, pr, nullptr, lds, C22,
                               lda, 1.f, true, nullptr, nullptr));
        }
    }
    return last_cuda(ctx);
}

// Right-looking mixed LU with partial pivoting and block b.
hdbf_status getrf_mixed_body(hdbf_context* ctx, int prec, float* A, long long lda, int n, int b,
                             int* ipiv, int* info, char* arena)
{
    const PrecInfo pi = prec_info(prec);
    if (pi.fmt < 0) return HDBF_STATUS_INVALID_VALUE;
    GetrfWs ws;
    HDBF_TRY(getrf_workspace(ctx, n, &ws));
    const long long lds = pad8(b);
    const size_t one = (size_t)n * lds * 2;
    void* hL = arena;
    void* hU = arena + one;
    void* lL = pi.split ? arena + 2 * one : nullptr;
    void* lU = pi.split ? arena + 3 * one : nullptr;
    void* scratch_lo = arena + 3 * one;
    const PrecInfo tp = trsm_prec(pi);
    const WBlock wb = w_block(arena, n, b);
    // |L| <= 1 under partial pivoting: L's shadow is unscaled; U's FP16 shadow
    // carries a per-panel power-of-two scale.
    unsigned* slots = reinterpret_cast<unsigned*>(arena + mixed_slots_offset(n, b));
    const bool scaled = pi.fmt == kFmtF16;
    if (info) cudaMemsetAsync(info, 0, sizeof(int), ctx->stream);
    for (int p = 0; p < n; p += b) {
        unsigned* slot = scaled ? slots + p / b : nullptr;
        const int psz = std::min(b, n - p);
        const int next = p + psz;
        const int tr = n - next;
        HDBF_TRY(getrf_panel(ctx, n - p, psz, at(A, lda, p, p), lda, ipiv + p, p, info, p, true,
                             ws));
        // this panel's row interchanges on every other column
        HDBF_TRY(compose_swaps(ctx, ipiv + p, psz, p, n - p, ws.src, ws.tgt, ws.count, ws.gperm,
                               info));
        const int max_moves = std::min(n - p, 2 * psz);
        if (p > 0)
            HDBF_TRY(apply_moves(ctx, at(A, lda, p, 0), lda, p, ws.src, ws.tgt, ws.count,
                                 max_moves, ws.temp, ws.temp_cols));
        if (tr <= 0) continue;
        HDBF_TRY(apply_moves(ctx, at(A, lda, p, next), lda, tr, ws.src, ws.tgt, ws.count,
                             max_moves, ws.temp, ws.temp_cols));
        // U12 = L11^{-1} A12 as one tensor-core GEMM: W = L11^{-1} (unit lower)
        // is the FP32 TRSM of the identity.
        float* A12 = at(A, lda, p, next);
        if (trsm_on_tc(pi)) {
            HDBF_TRY(set_identity(ctx, wb.W, wb.ldw, psz));
            HDBF_TRY(trsm_llu(ctx, psz, psz, at(A, lda, p, p), lda, wb.W, wb.ldw));
            HDBF_TRY(convert_transpose16(ctx, tp.fmt, psz, psz, wb.W, wb.ldw, wb.wh,
                                         tp.split ? wb.wl : nullptr, wb.ldws, 1.f));
            HDBF_TRY(convert_direct16(ctx, tp.fmt, psz, tr, A12, lda, hU,
                                      tp.split ? scratch_lo : nullptr, lds, 1.f));
            HDBF_TRY(zero_block(ctx, A12, lda, psz, tr));
            HDBF_TRY(tc_update(ctx, tp, psz, tr, psz, wb.wh, wb.wl, wb.ldws, hU, scratch_lo, lds,
                               A12, lda, -1.f, false));
        } else {
            HDBF_TRY(trsm_llu(ctx, psz, tr, at(A, lda, p, p), lda, A12, lda));
        }
        HDBF_TRY(convert_transpose16(ctx, pi.fmt, tr, psz, at(A, lda, next, p), lda, hL, lL, lds,
                                     1.f));
        if (slot) HDBF_TRY(panel_absmax(ctx, at(A, lda, p, next), lda, psz, tr, slot));
        HDBF_TRY(convert_direct16(ctx, pi.fmt, psz, tr, at(A, lda, p, next), lda, hU, lU, lds, 1.f,
                                  slot));
        HDBF_TRY(tc_update(ctx, pi, tr, tr, psz, hL, lL, lds, hU, lU, lds, at(A, lda, next, next),
                           lda, 1.f, false, nullptr, slot));
    }
    return last_cuda(ctx);
}

hdbf_status potrf_mixed(hdbf_context* ctx, int prec, float* A, long long lda, int n, int b,
                        int* info)
{
    if (n < 0 || (n > 0 && (!A || lda < n))) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0) return HDBF_STATUS_SUCCESS;
    const PrecInfo pi = prec_info(prec);
    if (pi.fmt < 0) return HDBF_STATUS_INVALID_VALUE;
    if (b <= 0) b = 512;
    b = std::min(b, n);
    HDBF_TRY(ensure_ws(ctx, n));
    hdbf_status st;
    char* arena = static_cast<char*>(mixed_arena(ctx, mixed_shadow_bytes(n, b, pi.split), &st));
    if (!arena) return st;
    ctx->mixed_fallbacks =
        trsm_on_tc(pi) ? reinterpret_cast<unsigned*>(arena + mixed_slots_offset(n, b)) +
                             2 * mixed_slot_words(n, b)
                       : nullptr;
    const std::vector<long long> key = {30, prec, (long long)A, lda, n, b, (long long)info,
                                        (long long)arena};
    return run_graph(ctx, key, [&] { return potrf_mixed_body(ctx, prec, A, lda, n, b, info, arena); });
}

hdbf_status getrf_mixed(hdbf_context* ctx, int prec, float* A, long long lda, int n, int b,
                        int* ipiv, int* info)
{
    if (n < 0 || (n > 0 && (!A || lda < n || !ipiv))) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0) return HDBF_STATUS_SUCCESS;
    const PrecInfo pi = prec_info(prec);
    if (pi.fmt < 0) return HDBF_STATUS_INVALID_VALUE;
    if (b <= 0) b = 512;
    b = std::min(b, n);
    HDBF_TRY(ensure_ws(ctx, n));
    hdbf_status st;
    char* arena = static_cast<char*>(mixed_arena(ctx, mixed_shadow_bytes(n, b, pi.split), &st));
    if (!arena) return st;
    const std::vector<long long> key = {31, prec, (long long)A, lda, n, b, (long long)ipiv,
                                        (long long)info, (long long)arena};
    return run_graph(ctx, key, [&] {
        return getrf_mixed_body(ctx, prec, A, lda, n, b, ipiv, info, arena);
    });
}

}  // namespace hdbf

using namespace hdbf;

extern "C" {

hdbf_status hdbf_spotrf_mixed(hdbf_handle h, hdbf_precision prec, float* A, int lda, int n, int nb,
                              int* info)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = potrf_mixed(h, (int)prec, A, lda, n, nb, info);
}

hdbf_status hdbf_mixed_fallback_panels(hdbf_handle h, int* count)
{
    if (!h || !count) return h ? HDBF_STATUS_INVALID_VALUE : HDBF_STATUS_INVALID_HANDLE;
    *count = 0;
    if (!h->mixed_fallbacks) return HDBF_STATUS_SUCCESS;
    unsigned v = 0;
    if (cudaMemcpyAsync(&v, h->mixed_fallbacks, sizeof(v), cudaMemcpyDeviceToHost, h->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    *count = (int)v;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_sgetrf_mixed(hdbf_handle h, hdbf_precision prec, float* A, int lda, int n, int nb,
                              int* ipiv, int* info)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = getrf_mixed(h, (int)prec, A, lda, n, nb, ipiv, info);
}

// Reference recursive_potrf_mixed_driver (src/potrf/recursive_potrf.cpp:
// 350-388): FP16 products with the reference's damping retry at failure
// (lambda0 = 1e-4 * max|a_ii| -- 6.55 on the reference's 65504-scaled
// matrix --, doubled, at most 5 attempts).  The FP16 range is handled by the
// shadow scale, so the matrix itself is not rescaled.
void recursive_potrf_mixed_driver(hdbf_handle h, StreamPool* pool, float* A, int lda, int n,
                                  int nb, int* info)
{
    (void)pool;
    if (!h) return;
    if (n < 0 || (n > 0 && (!A || lda < n))) { h->last_status = HDBF_STATUS_INVALID_VALUE; return; }
    if (n == 0) { h->last_status = HDBF_STATUS_SUCCESS; return; }
    const size_t bytes = (size_t)n * n * sizeof(float);
    hdbf_status st = ensure_ws(h, n);
    if (st != HDBF_STATUS_SUCCESS) { h->last_status = st; return; }
    float maxdiag = 0.f;
    st = absmax_host(h, A, lda, n, n, true, &maxdiag);
    if (st != HDBF_STATUS_SUCCESS) { h->last_status = st; return; }
    // Backup of A for the damping retries (kept out of the mixed arena,
    // which the factorization uses for its shadows).
    float* backup = nullptr;
    if (cudaMalloc(&backup, bytes) != cudaSuccess) {
        cudaGetLastError();
        h->last_status = HDBF_STATUS_ALLOC_FAILED;
        return;
    }
    cudaMemcpy2DAsync(backup, (size_t)n * 4, A, (size_t)lda * 4, (size_t)n * 4, n,
                      cudaMemcpyDeviceToDevice, h->stream);
    float lambda = 1e-4f * maxdiag;
    for (int attempt = 0; attempt <= 5; ++attempt) {
        if (attempt > 0) {
            cudaMemcpy2DAsync(A, (size_t)lda * 4, backup, (size_t)n * 4, (size_t)n * 4, n,
                              cudaMemcpyDeviceToDevice, h->stream);
            launch_add_damping(A, n, lda, lambda, h->stream);
            lambda *= 2.f;
        }
        st = potrf_mixed(h, HDBF_PREC_FP16, A, lda, n, nb > 0 ? nb : 512, info);
        if (st != HDBF_STATUS_SUCCESS) break;
        int hinfo = 0;
        cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        cudaStreamSynchronize(h->stream);
        if (hinfo <= 0) break;
    }
    cudaStreamSynchronize(h->stream);
    cudaFree(backup);
    h->last_status = st;
}

void batched_syrk_bottom_up_mixed(hdbf_handle h, StreamPool* pool, float* A, int lda, float* C,
                                  int ldc, int n, int k, int nb)
{
    (void)pool;
    (void)nb;
    if (!h) return;
    if (n <= 0 || k <= 0) { h->last_status = HDBF_STATUS_SUCCESS; return; }
    if (!A || !C || lda < n || ldc < n) { h->last_status = HDBF_STATUS_INVALID_VALUE; return; }
    const long long kp = pad8(k);
    hdbf_status st;
    char* arena = static_cast<char*>(mixed_arena(h, (size_t)n * kp * 2 + 256, &st));
    if (!arena) { h->last_status = st; return; }
    const PrecInfo pi = {kFmtF16, false};
    st = convert_transpose16(h, kFmtF16, n, k, A, lda, arena, nullptr, kp, 1.f);
    if (st == HDBF_STATUS_SUCCESS)
        st = tc_update(h, pi, n, n, k, arena, nullptr, kp, arena, nullptr, kp, C, ldc, 1.f, true);
    h->last_status = st;
}

// B (n x m) <- B * A^{-T}: recursion on column halves down to nb (FP32
// leaves), the update B2 -= X1 L21^T on FP16 tensor cores.
static hdbf_status rec_trsm_mixed(hdbf_context* ctx, const float* L, long long ldl, float* B,
                                  long long ldb, int n, int m, int nb, char* arena)
{
    if (n <= 0 || m <= 0) return HDBF_STATUS_SUCCESS;
    if (m <= nb || nb <= 0) return trsm_rlt(ctx, n, m, L, ldl, B, ldb);
    const int m1 = m / 2, m2 = m - m1;
    HDBF_TRY(rec_trsm_mixed(ctx, L, ldl, B, ldb, n, m1, nb, arena));
    const long long kp = pad8(m1);
    void* xs = arena;
    void* ls = arena + (size_t)n * kp * 2;
    HDBF_TRY(convert_transpose16(ctx, kFmtF16, n, m1, B, ldb, xs, nullptr, kp, 1.f));
    HDBF_TRY(convert_transpose16(ctx, kFmtF16, m2, m1, L + m1, ldl, ls, nullptr, kp, 1.f));
    const PrecInfo pi = {kFmtF16, false};
    HDBF_TRY(tc_update(ctx, pi, n, m2, m1, xs, nullptr, kp, ls, nullptr, kp, B + (long long)m1 * ldb,
                       ldb, 1.f, false));
    return rec_trsm_mixed(ctx, L + (long long)m1 * ldl + m1, ldl, B + (long long)m1 * ldb, ldb, n,
                          m2, nb, arena);
}

void recursive_trsm_mixed(hdbf_handle h, float* A, int lda, float* B, int ldb, int n, int m, int nb)
{
    if (!h) return;
    if (n <= 0 || m <= 0) { h->last_status = HDBF_STATUS_SUCCESS; return; }
    if (!A || !B || lda < m || ldb < n) { h->last_status = HDBF_STATUS_INVALID_VALUE; return; }
    hdbf_status st = ensure_ws(h, std::max(n, m));
    if (st != HDBF_STATUS_SUCCESS) { h->last_status = st; return; }
    const size_t need = (size_t)(n + m) * pad8(m) * 2 + 1024;
    char* arena = static_cast<char*>(mixed_arena(h, need, &st));
    if (!arena) { h->last_status = st; return; }
    h->last_status = rec_trsm_mixed(h, A, lda, B, ldb, n, m, nb, arena);
}

}  // extern "C"
