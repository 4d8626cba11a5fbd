// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "hdbf/hdbf.h"

namespace hdbf {
// Kernel classes for the per-launch event profiler (hdbf_profile_*).
enum KernelClass {
    kClsGemm = 0,     // sgemm_sub_kernel (GEMM / SYRK trailing updates)
    kClsPotf2 = 1,    // potf2_kernel
    kClsTrsmR = 2,    // trsm_rlt_kernel
    kClsTrsmL = 3,    // trsm_llu_kernel
    kClsPanel = 4,    // getf2_coop_kernel
    kClsCompose = 5,  // compose_swaps_kernel
    kClsMoves = 6,    // apply_moves kernels
    kClsOther = 7,
    kNumClasses = 8
};
struct ProfRec {
    int cls;
    cudaEvent_t a, b;
    double flops;
    double bytes;
};
}  // namespace hdbf

struct hdbf_context {
    cudaStream_t stream = nullptr;
    int device = 0;
    int sm_count = 148;
    size_t max_smem_optin = 0;
    // Workspace arena (grown on demand outside stream capture).
    void* ws = nullptr;
    size_t ws_bytes = 0;
    // Small always-present device block: [0] error word, [1..] barrier words.
    int* dev_small = nullptr;
    hdbf_status last_status = HDBF_STATUS_SUCCESS;
    unsigned long long launches = 0;
    // Optional per-launch event profiling.
    bool profiling = false;
    std::vector<hdbf::ProfRec> prof;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
};

struct hdbf_stream_pool {
    cudaStream_t* streams = nullptr;
    int count = 0;
};

namespace hdbf {

// Layout of hdbf_context::dev_small (ints).
constexpr int kSmallErr = 0;       // device error word (timeouts, invalid pivots)
constexpr int kSmallBarCount = 4;  // grid-barrier arrive counter
constexpr int kSmallBarGen = 8;    // grid-barrier generation
constexpr int kSmallMoveCount = 12;  // move count of the last composed permutation
constexpr int kSmallInts = 64;

// Device error codes written into dev_small[kSmallErr].
constexpr int kErrTimeout = 1;
constexpr int kErrBadPivot = 2;

// Bounded-wait poll limit for grid barriers (~0.5 s with back-off).
constexpr unsigned kSpinLimit = 1u << 22;

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// RAII: when profiling is on, brackets one launch with a pair of events on
// ctx->stream and records its class and algorithmic work.
class ProfScope {
public:
    ProfScope(hdbf_context* ctx, int cls, double flops, double bytes = 0.0);
    ~ProfScope();
private:
    hdbf_context* ctx_;
    int idx_ = -1;
};

// Make sure the workspace holds at least `bytes`; returns nullptr and sets
// *st on failure.  Growing frees the old buffer (device-synchronising).
void* workspace(hdbf_context* ctx, size_t bytes, hdbf_status* st);

hdbf_status last_cuda(hdbf_context* ctx);

// ---------------------------------------------------------------- kernels
// All launchers enqueue on ctx->stream and count launches.

// C(M x N) -= A(M x K) * op(B); op(B) = B^T (B is N x K, nn=false) or B
// (B is K x N, nn=true).  lower_only: tiles wholly above the diagonal are
// skipped and only entries with row >= col (local to C) are written.
hdbf_status sgemm_sub(hdbf_context* ctx, bool nn, bool lower_only, int M, int N, int K,
                      const float* A, long long lda, const float* B, long long ldb,
                      float* C, long long ldc);

// Unblocked-in-shared-memory Cholesky of an n x n (n <= 64) diagonal block.
hdbf_status potf2_small(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                        int info_base);

// B(rows x cols) <- B * L^{-T}, L lower non-unit, cols <= 64.
hdbf_status trsm_rlt_small(hdbf_context* ctx, int rows, int cols, const float* L,
                           long long ldl, float* B, long long ldb);
// B(rows x cols) <- L^{-1} B, L unit lower, rows <= 64.
hdbf_status trsm_llu_small(hdbf_context* ctx, int rows, int cols, const float* L,
                           long long ldl, float* B, long long ldb);

// Cooperative partially pivoted LU of an m x w panel (w <= 32).  Pivots are
// written 1-based as (local row + 1 + ipiv_add).
hdbf_status getf2_coop(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                       int ipiv_add, int* info, int info_base, bool pivot);
size_t getf2_coop_scratch_bytes();

// Compose LAPACK swaps  row (i) <-> row (ipiv[i]-1-ipiv_minus), i in [0,k),
// over local rows [0, m) into (src, tgt, *count) moves.
hdbf_status compose_swaps(hdbf_context* ctx, const int* ipiv, int k, int ipiv_minus, int m,
                          int* src, int* tgt, int* count, int* gperm, int* info);
// A[tgt[i], c] = old A[src[i], c] for c < ncols, i < *count (<= max_moves).
hdbf_status apply_moves(hdbf_context* ctx, float* A, long long lda, int ncols,
                        const int* src, const int* tgt, const int* count, int max_moves,
                        float* temp, long long temp_cols);

// Auxiliary kernels.
hdbf_status fill_uniform(hdbf_context* ctx, float* x, size_t count, uint64_t seed,
                         uint64_t offset);
hdbf_status add_damping(cudaStream_t s, float* A, int n, long long lda, float lambda);

// ---------------------------------------------------------------- drivers
hdbf_status potrf_diag(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                       int info_base);
hdbf_status trsm_rlt(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                     float* B, long long ldb);
hdbf_status trsm_llu(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                     float* B, long long ldb);
hdbf_status syrk_lower(hdbf_context* ctx, int n, int k, const float* A, long long lda,
                       float* C, long long ldc);
struct GetrfWs {
    int* src = nullptr;    // composed move sources (n ints)
    int* tgt = nullptr;    // composed move targets (n ints)
    int* count = nullptr;  // device move count
    int* gperm = nullptr;  // global permutation scratch (n ints) for very tall panels
    float* temp = nullptr;  // column-tiled swap buffer
    long long temp_cols = 0;
};
// Carve the factorization workspace for order n (reserves it first).
hdbf_status getrf_workspace(hdbf_context* ctx, int n, GetrfWs* ws);
hdbf_status getrf_panel(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                        int ipiv_add, int* info, int info_base, bool pivot, const GetrfWs& ws);

}  // namespace hdbf

#define HDBF_TRY(expr)                                   \
    do {                                                 \
        hdbf_status _st = (expr);                        \
        if (_st != HDBF_STATUS_SUCCESS) return _st;      \
    } while (0)
