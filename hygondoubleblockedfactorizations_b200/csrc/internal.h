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
    kClsTrsmR = 2,    // rlt_apply_kernel
    kClsTrsmL = 3,    // llu_apply_kernel
    kClsPanel = 4,    // getf2_cluster_kernel / getf2_coop_kernel
    kClsCompose = 5,  // compose_swaps_kernel
    kClsMoves = 6,    // apply_moves kernels
    kClsTrsmInv = 7,  // tri_inv64_kernel
    kClsTcGemm = 8,   // tc_gemm_persistent_kernel / tc_gemm_sub_kernel (tcgen05 updates)
    kClsConvert = 9,  // FP32 -> 16-bit shadow conversions
    kClsIr = 10,      // FP64 residual / update / norm kernels
    kClsOther = 11,
    kClsWave = 12,     // trsv_wave_kernel (wavefront triangular solves)
    kClsSkinny = 13,   // skinny_kernel (updates with N <= 32)
    kClsBatched = 14,  // batched_factor_solve_kernel
    kClsSelector = 15, // selector MLP kernels
    kClsPotrfBlock = 16, // potrf_block_kernel (cooperative diagonal-block Cholesky)
    kNumClasses = 17
};
// Algorithm stages of the double-blocked drivers for the per-stage profile
// (hdbf_profile_stages), named as the reference's stage profilers name them
// (src/potrf/profile_double_blocked_potrf.cpp, src/getrf/getrf_batched_pivot_internal.h).
enum Stage {
    kStNone = 0,
    kStPotrf,            // "POTRF": diagonal-block Cholesky
    kStTrsm,             // "TRSM": panel TRSM of the Cholesky
    kStInnerGemm,        // "Inner GEMM"
    kStOuterSyrk,        // "Outer SYRK"
    kStOuterGemm,        // "Outer GEMM"
    kStPanel,            // "Panel GETRF"
    kStPivotProp,        // "Pivot propagation" (immediate pivoting)
    kStInnerPivot,       // "Inner pivot batch"
    kStInnerTrsm,        // "Inner TRSM"
    kStOuterPivot,       // "Outer pivot batch"
    kStOuterTrsmBlock,   // "Outer TRSM block"
    kStOuterTrsmGemm,    // "Outer TRSM GEMM"
    kStOuterTrsmDirect,  // "Outer TRSM direct"
    kNumStages
};
struct ProfRec {
    int cls;
    cudaEvent_t a, b;
    double flops;
    double bytes;
    int m = 0, n = 0, k = 0;  // problem shape (GEMM launches)
    int stage = 0;            // Stage active when the launch was enqueued
    unsigned call = 0;        // which entry into that stage (StageScope instance)
};
struct GraphEntry {
    std::vector<long long> key;
    cudaGraphExec_t exec = nullptr;
    std::vector<ProfRec> prof;  // event pairs baked into the graph (profiling graphs)
    unsigned long long id = 0;
    unsigned long long last_use = 0;
    unsigned long long kernels = 0;  // kernel launches recorded in the graph
};
}  // namespace hdbf

namespace hdbf {
constexpr int kLaEvents = 33;  // 32 outer-update chunks per block + the join
}

struct hdbf_context {
    cudaStream_t stream = nullptr;
    int device = 0;
    int sm_count = 148;
    size_t max_smem_optin = 0;
    int cluster_max = 0;  // largest cluster the panel kernel can launch (0: none)
    int panel_mode = 0;   // hdbf_set_panel_kernel
    int panel_leaf = 128; // GETRF panel recursion leaf width (32, 64 or 128)
    int panel_rows = 256; // target rows per CTA of the grid-wide panel kernel
    // GETRF look-ahead (hdbf_set_lookahead): the panel chain of an outer block
    // runs on a high-priority internal stream while the caller's stream still
    // applies the outer update chunk by chunk; la_ev[c] marks chunk c done and
    // la_ev[kLaEvents - 1] joins the panel chain back.
    int lookahead = 1;
    cudaStream_t la_stream = nullptr;
    cudaEvent_t la_ev[hdbf::kLaEvents] = {};
    bool la_used = false;    // the graph being captured forked onto la_stream
    bool no_skinny = false;  // keep GEMMs off the shared split-K scratch
    // K chunk of the FP32 GEMM split (SplitPlan): -1 decides per launch,
    // 0 never splits, > 0 splits K into chunks of this many.  Column chunks of
    // one GEMM take the whole GEMM's plan so their sums match it bit for bit.
    int split_kc = -1;
    // Tensor-core GEMM kernel: 0 persistent 128 x 256 tiles with two TMEM
    // accumulators (default), 1 one 128 x 128 tile per CTA (HDBF_TC_KERNEL).
    int tc_kernel = 0;
    unsigned spin_limit = 0; // hdbf_set_wait_limit (0: default)
    // Conditional launches (RunIf): while set, the FP32 GEMM and the
    // diagonal-block kernel run only when *run_if != 0 (read on the device).
    const int* run_if = nullptr;
    // Device counter of panels the last mixed Cholesky rebuilt in FP32.
    unsigned* mixed_fallbacks = nullptr;
    // Stage attribution of profiled launches (StageScope) and the per-stage
    // split of the last profiling interval (hdbf_profile_stages).
    int stage = 0;
    unsigned stage_call = 0, stage_seq = 0;
    double stage_ms[32] = {}, stage_flops[32] = {};
    int stage_calls[32] = {};
    // Workspace arena (grown on demand outside stream capture).
    void* ws = nullptr;
    size_t ws_bytes = 0;
    int ws_n = 0;  // largest order whose layout fits in ws_bytes
    // Small always-present device block: [0] error word, [1..] barrier words.
    int* dev_small = nullptr;
    // Second arena for the mixed-precision path (16-bit shadows, FP64 IR
    // vectors); grown on demand outside stream capture.
    void* mix = nullptr;
    size_t mix_bytes = 0;
    hdbf_status last_status = HDBF_STATUS_SUCCESS;
    unsigned long long launches = 0;
    // Optional per-launch event profiling.
    bool profiling = false;
    std::vector<hdbf::ProfRec> prof;
    // CUDA-graph cache of whole factorizations (key = entry point + arguments).
    bool use_graphs = true;
    bool capturing = false;
    cudaStream_t cap_stream = nullptr;
    std::vector<hdbf::GraphEntry> graphs;
    unsigned long long graph_clock = 0;
    std::vector<unsigned long long> prof_graph_ids;  // graphs replayed while profiling
};

struct hdbf_stream_pool {
    cudaStream_t* streams = nullptr;
    int count = 0;
};

namespace hdbf {

// Layout of hdbf_context::dev_small (ints).
constexpr int kSmallErr = 0;       // device error word (timeouts, invalid pivots)
constexpr int kSmallSpin = 8;        // bounded-wait poll limit of the handle (0: kSpinLimit)
constexpr int kSmallMoveCount = 12;  // move count of the last composed permutation
constexpr int kSmallEpoch = 16;      // panel-kernel exchange epoch
constexpr int kSmallDone = 20;       // panel-kernel finished-CTA counter
constexpr int kSmallScratch = 24;    // host-read reduction results (absmax etc.)
constexpr int kSmallBlockBar = 32;   // diagonal-block kernel: barrier counter, fail, abort
constexpr int kSmallInts = 64;

// Device error codes written into dev_small[kSmallErr]; the first error
// recorded stays (atomicCAS from 0) until hdbf_check_device_errors reads it.
constexpr int kErrTimeout = 1;
constexpr int kErrBadPivot = 2;

// Default bounded-wait poll limit for grid barriers (~0.5 s with back-off).
constexpr unsigned kSpinLimit = 1u << 22;

#ifdef __CUDACC__
// Per-panel power-of-two scale of the 16-bit shadows, from the panel's max |x|
// given as FP32 bits (written by an atomicMax over the panel): s = 2^k with
// max * s in [128, 256); 1 for a zero or non-finite max; k clamped to
// [-60, 60].  Exact (built from the exponent bits), so the converting kernel
// and the GEMM epilogue that undoes it agree bit for bit.
__device__ __forceinline__ int panel_scale_exp(unsigned maxbits)
{
    const int e = (int)((maxbits >> 23) & 0xffu);
    if (maxbits == 0u || e == 0xff) return 0;
    const int k = e == 0 ? 60 : 7 - (e - 127);
    return k < -60 ? -60 : (k > 60 ? 60 : k);
}
__device__ __forceinline__ float pow2f_exact(int k)
{
    return __uint_as_float((unsigned)(127 + k) << 23);
}

// The handle's poll limit, read at kernel start from the small device block
// whose error word `err` points at (hdbf_set_wait_limit).
__device__ __forceinline__ unsigned spin_limit_of(const int* err)
{
    const unsigned v = *reinterpret_cast<const volatile unsigned*>(err + (kSmallSpin - kSmallErr));
    return v ? v : kSpinLimit;
}
#endif

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// RAII: when profiling is on, brackets one launch with a pair of events on
// ctx->stream and records its class and algorithmic work.
class ProfScope {
public:
    ProfScope(hdbf_context* ctx, int cls, double flops, double bytes = 0.0, int m = 0,
              int n = 0, int k = 0);
    ~ProfScope();
private:
    hdbf_context* ctx_;
    int idx_ = -1;
};

// RAII: launches enqueued while it lives are attributed to `stage` (one
// "call" of that stage per scope).
class StageScope {
public:
    StageScope(hdbf_context* ctx, int stage)
        : ctx_(ctx), prev_(ctx->stage), prev_call_(ctx->stage_call)
    {
        ctx->stage = stage;
        ctx->stage_call = ++ctx->stage_seq;
    }
    ~StageScope()
    {
        ctx_->stage = prev_;
        ctx_->stage_call = prev_call_;
    }
private:
    hdbf_context* ctx_;
    int prev_;
    unsigned prev_call_;
};

// RAII: launches of the conditional-capable kernels (FP32 GEMM, diagonal-block
// Cholesky, block-column restore) enqueued while it lives do their work only
// if *flag != 0 when they run; the skinny GEMM path is not taken meanwhile.
class RunIf {
public:
    RunIf(hdbf_context* ctx, const int* flag) : ctx_(ctx), prev_(ctx->run_if) { ctx->run_if = flag; }
    ~RunIf() { ctx_->run_if = prev_; }
private:
    hdbf_context* ctx_;
    const int* prev_;
};

// Make sure the workspace holds at least `bytes`; returns nullptr and sets
// *st on failure.  Growing frees the old buffer (device-synchronising).
void* workspace(hdbf_context* ctx, size_t bytes, hdbf_status* st);

// Mixed-path arena of at least `bytes` (same growth rules as the workspace).
void* mixed_arena(hdbf_context* ctx, size_t bytes, hdbf_status* st);

// Workspace layout for problems of order <= n (byte offsets):
//   coop  panel-kernel exchange slots (fixed size, offset 0)
//   inv   inverted 64x64 diagonal blocks, ceil(n/64)*4096 floats
//   perm  running composed row permutation of a GETRF outer block, n ints
//   coop64  FP64 panel-kernel exchange slots (fixed size)
//   src, tgt, gperm  composed row moves / permutation scratch, n ints each
//   temp  column-tiled swap buffer, 64*n floats
//   skinny  split-K partial sums of the skinny GEMM, 256*n floats
//   wave  wavefront-solve row-major x copy (32 columns) and its flags
struct WsLayout {
    size_t coop, inv, perm, coop64, src, tgt, gperm, temp, skinny, wave, split, total;
};
// Split-K partial sums of under-filled FP32 GEMM launches: two halves of
// kSplitFloats each, one for the handle's stream and one for its look-ahead
// stream, so concurrent GEMMs on the two never share scratch.
constexpr size_t kSplitFloats = (size_t)32 << 20;
WsLayout ws_layout(int n);
// Guarantee the layout for order n (grows the arena outside stream capture).
hdbf_status ensure_ws(hdbf_context* ctx, int n);
float* ws_coop(hdbf_context* ctx);
float* ws_inv(hdbf_context* ctx);
int* ws_perm(hdbf_context* ctx);
double* ws_coop64(hdbf_context* ctx);
int* ws_src(hdbf_context* ctx);
int* ws_tgt(hdbf_context* ctx);
int* ws_gperm(hdbf_context* ctx);
float* ws_temp(hdbf_context* ctx);
float* ws_skinny(hdbf_context* ctx);
// Split-K scratch half for GEMMs enqueued on ctx->stream.
float* ws_split(hdbf_context* ctx);
float* ws_wave(hdbf_context* ctx);

hdbf_status last_cuda(hdbf_context* ctx);

// ---------------------------------------------------------------- kernels
// All launchers enqueue on ctx->stream and count launches.

// C(M x N) -= A(M x K) * op(B); op(B) = B^T (B is N x K, nn=false) or B
// (B is K x N, nn=true).  lower_only: tiles wholly above the diagonal are
// skipped and only entries with row >= col (local to C) are written.
hdbf_status sgemm_sub(hdbf_context* ctx, bool nn, bool lower_only, int M, int N, int K,
                      const float* A, long long lda, const float* B, long long ldb,
                      float* C, long long ldc);

// K split of the FP32 GEMM of shape M x N x K (tri: lower-triangle mode):
// the number of chunks (1 = no split) and, in *kc, their length.
int split_count(const hdbf_context* ctx, int M, int N, int K, bool tri, int* kc);
// While alive, every FP32 GEMM splits K as the GEMM of the given shape does.
struct SplitPlan {
    hdbf_context* ctx;
    int saved;
    SplitPlan(hdbf_context* c, int M, int N, int K) : ctx(c), saved(c->split_kc)
    {
        int kc = 0;
        const int S = split_count(c, M, N, K, false, &kc);
        c->split_kc = S > 1 ? kc : 0;
    }
    ~SplitPlan() { ctx->split_kc = saved; }
};

// Skinny update (N <= 32): mode 0 C -= A * B^T, 1 C -= A * B, 2 C -= A^T * B,
// with the operand shapes of sgemm_sub / sgemm_sub_tn.  sgemm_launch routes
// narrow non-triangular updates here.
hdbf_status sgemm_skinny(hdbf_context* ctx, int mode, int M, int N, int K, const float* A,
                         long long lda, const float* B, long long ldb, float* C, long long ldc);
size_t skinny_partial_floats(int n);

// C(M x N) -= A^T * B with A stored K x M and B stored K x N (column-major).
hdbf_status sgemm_sub_tn(hdbf_context* ctx, int M, int N, int K, const float* A, long long lda,
                         const float* B, long long ldb, float* C, long long ldc);

// Unblocked-in-shared-memory Cholesky of an n x n (n <= 64) diagonal block.
hdbf_status potf2_small(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                        int info_base);

// Inverses of the 64x64 diagonal blocks of lower-triangular L (order n) into
// out[b*4096 ...] (column-major blocks); unit selects an implicit unit diagonal.
hdbf_status tri_inv64(hdbf_context* ctx, int n, const float* L, long long ldl, bool unit,
                      float* out);
// Leaf applications of a precomputed block inverse (in place):
// B(rows<=64 x cols) <- inv * B  and  B(rows x cols<=64) <- B * inv^T.
hdbf_status llu_apply(hdbf_context* ctx, int rows, int cols, const float* inv, float* B,
                      long long ldb);
hdbf_status rlt_apply(hdbf_context* ctx, int rows, int cols, const float* inv, float* B,
                      long long ldb);

// Inverse modes: 0 lower non-unit, 1 lower unit, 2 upper non-unit.
hdbf_status tri_inv64_mode(hdbf_context* ctx, int n, const float* L, long long ldl, int mode,
                           float* out);
// B(rows <= 256 x cols) <- L^{-1} B for unit lower L in one launch (block
// forward substitution with the 64x64 inverses in inv, trsm_block.cu).
hdbf_status llu_block(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                      const float* inv, float* B, long long ldb);
int llu_block_max_rows();
// B(rows x cols <= 256) <- B L^{-T}, L lower non-unit, same scheme.
hdbf_status rlt_block(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                      const float* inv, float* B, long long ldb);
void configure_trsm_block_kernels(hdbf_context* ctx);
// B <- inv * B (trans=false) or inv^T * B (trans=true), rows <= 64.
hdbf_status llu_apply_t(hdbf_context* ctx, int rows, int cols, const float* inv, float* B,
                        long long ldb, bool trans);

// Solves on FP32 factors (solves.cu).
hdbf_status ipiv_to_perm(hdbf_context* ctx, const int* ipiv, int n, int* perm);
hdbf_status gather_rows_perm(hdbf_context* ctx, const float* src, long long lds, float* dst,
                             long long ldd, const int* perm, int n, int cols);
hdbf_status potrs_f32(hdbf_context* ctx, const float* L, long long ldl, int n, int nrhs, float* B,
                      long long ldb);
hdbf_status getrs_f32_permuted(hdbf_context* ctx, const float* LU, long long ldlu, int n, int nrhs,
                               float* B, long long ldb);
void configure_solve_kernels(hdbf_context* ctx);

// Wavefront block triangular solve (trsm_wave.cu): B <- op(M)^{-1} B, M = T
// (trans false) or T^T (trans true); forward for a lower M, backward for an
// upper one.  inv holds the 64x64 diagonal-block inverses of T from
// tri_inv64_mode (applied transposed when trans is set).  One launch per 32
// right-hand-side columns.
hdbf_status trsv_wave(hdbf_context* ctx, int n, int nrhs, const float* T, long long ldt, bool trans,
                      const float* inv, bool backward, float* B, long long ldb);
size_t wave_scratch_bytes(int n);
void configure_wave_kernels(hdbf_context* ctx);
void configure_batched_kernels(hdbf_context* ctx);

// Cooperative partially pivoted LU of an m x w panel (w <= 128).  Pivots are
// written 1-based as (local row + 1 + ipiv_add).
hdbf_status getf2_coop(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                       int ipiv_add, int* info, int info_base, bool pivot);
size_t getf2_coop_scratch_bytes();
void configure_getrf_kernels(hdbf_context* ctx);
// Same contract on one thread-block cluster with the block in distributed
// shared memory; NOT_SUPPORTED when the block does not fit (caller falls
// back to getf2_coop).
hdbf_status getf2_cluster(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                          int ipiv_add, int* info, int info_base, bool pivot);
int configure_cluster_panel(hdbf_context* ctx);

// Compose LAPACK swaps  row (i) <-> row (ipiv[i]-1-ipiv_minus), i in [0,k),
// over local rows [0, m) into (src, tgt, *count) moves (at most 2k): rows
// [0, k) in order, then the distinct pivot rows >= k in increasing order.
// k <= 4096 runs without replaying the swaps (sorted-group composition, O(k)
// rows touched); longer sequences are replayed by one thread over perm[m]
// (gperm when m ints do not fit in shared memory).
hdbf_status compose_swaps(hdbf_context* ctx, const int* ipiv, int k, int ipiv_minus, int m,
                          int* src, int* tgt, int* count, int* gperm, int* info);
// A[tgt[i], c] = old A[src[i], c] for c < ncols, i < *count (<= max_moves).
// Running composition: pos (m ints, row i of the block holds original row
// pos[i]) is reset to the identity when init is set, then the LAPACK swaps
// ipiv[k0, k1) (1-based, minus ipiv_minus gives rows local to the block) are
// composed onto it, and every i with pos[i] != i becomes a move (pos[i] -> i),
// in increasing i.  Fails (count 0, info -1) on a pivot outside [i, m).
hdbf_status compose_running(hdbf_context* ctx, const int* ipiv, int k0, int k1, int ipiv_minus,
                            int m, int* pos, bool init, int* src, int* tgt, int* count,
                            int* info);
// Whether compose_running takes a block of height m and kk new swaps (its
// shared memory holds pos[m] and the sorted-group arrays; kk <= 4096).
bool compose_running_fits(hdbf_context* ctx, int m, int kk);
hdbf_status apply_moves(hdbf_context* ctx, float* A, long long lda, int ncols,
                        const int* src, const int* tgt, const int* count, int max_moves,
                        float* temp, long long temp_cols);

// ------------------------------------------------ tensor-core (tcgen05) path
// A K-major 16-bit operand: row r, element k at base[(row0 + r) * ld + k0 + k].
struct TcOperand {
    const void* base = nullptr;
    long long ld = 0;  // elements; multiple of 8
    int row0 = 0;
    int k0 = 0;        // multiple of 8
};
constexpr int kFmtF16 = 0;   // IEEE binary16
constexpr int kFmtBF16 = 1;  // bfloat16
// C(M x N, FP32 column-major) -= scale * A * B^T on the tensor cores.
// Optional device scales (sa_max / sb_max: panel max bits, see
// panel_scale_exp): the epilogue then uses scale / (s_a s_b).
hdbf_status tc_gemm_sub(hdbf_context* ctx, int fmt, int M, int N, int K, const TcOperand& A,
                        const TcOperand& B, float* C, long long ldc, float scale, bool lower_only,
                        const unsigned* sa_max = nullptr, const unsigned* sb_max = nullptr);
// C -= scale * (A B^T + A Blo^T + Alo B^T): the split-precision product in one
// launch (hi/lo operands share row/K origins), one FP32 accumulator in TMEM.
hdbf_status tc_gemm_sub_split(hdbf_context* ctx, int fmt, int M, int N, int K, const TcOperand& A,
                              const TcOperand& Alo, const TcOperand& B, const TcOperand& Blo,
                              float* C, long long ldc, float scale, bool lower_only,
                              const unsigned* sa_max = nullptr, const unsigned* sb_max = nullptr);
void configure_tc_kernels(hdbf_context* ctx);
// dst(r, k) = round16(s * src(r, k)) for an rows x cols FP32 column-major block
// into a K-major (row-major, ldd elements) 16-bit block; `hi_lo` additionally
// writes the rounding residual round16(s*src - hi) into lo (may be null).
// smax (optional): device max bits of the panel; the scale is then
// 2^panel_scale_exp(*smax) instead of s.
hdbf_status convert_transpose16(hdbf_context* ctx, int fmt, int rows, int cols, const float* src,
                                long long lds, void* hi, void* lo, long long ldd, float s,
                                const unsigned* smax = nullptr);
// dst[c * ldd + r] = round16(s * src[c * lds + r]): same layout (column-major
// FP32 -> "column = K-major row" 16-bit), with optional residual.
hdbf_status convert_direct16(hdbf_context* ctx, int fmt, int rows, int cols, const float* src,
                             long long lds, void* hi, void* lo, long long ldd, float s,
                             const unsigned* smax = nullptr);
// *slot = FP32 bits of max |A(r, c)| over rows x cols (slot cleared first).
hdbf_status panel_absmax(hdbf_context* ctx, const float* A, long long lda, int rows, int cols,
                         unsigned* slot);

// Auxiliary kernels.
hdbf_status fill_uniform(hdbf_context* ctx, float* x, size_t count, uint64_t seed,
                         uint64_t offset);
hdbf_status add_damping(cudaStream_t s, float* A, int n, long long lda, float lambda);

// ---------------------------------------------------------------- drivers
// Cholesky of an n x n (n <= potrf_block_max_n()) diagonal block in one
// cooperative launch; with W non-null also W = L^{-1} (lower, upper zeroed).
hdbf_status potrf_block(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                        int info_base, float* W, long long ldw);
int potrf_block_max_n();
hdbf_status potrf_diag(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                       int info_base);
hdbf_status trsm_rlt(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                     float* B, long long ldb);
hdbf_status trsm_llu(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                     float* B, long long ldb);
// Create the look-ahead stream and events (outside stream capture).
hdbf_status ensure_lookahead(hdbf_context* ctx);
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

// ---------------------------------------------------------------- FP64
// Overloads of the primitives above for the `_double` entry points
// (fp64.cu).  The FP64 workspace is the FP32 layout of order 2n.
inline hdbf_status gemm_sub(hdbf_context* ctx, bool nn, bool lower_only, int M, int N, int K,
                            const float* A, long long lda, const float* B, long long ldb,
                            float* C, long long ldc)
{
    return sgemm_sub(ctx, nn, lower_only, M, N, K, A, lda, B, ldb, C, ldc);
}
hdbf_status gemm_sub(hdbf_context* ctx, bool nn, bool lower_only, int M, int N, int K,
                     const double* A, long long lda, const double* B, long long ldb, double* C,
                     long long ldc);
hdbf_status gemm_sub_tn(hdbf_context* ctx, int M, int N, int K, const double* A, long long lda,
                        const double* B, long long ldb, double* C, long long ldc);
hdbf_status potf2_small(hdbf_context* ctx, int n, double* A, long long lda, int* info,
                        int info_base);
hdbf_status trsm_rlt(hdbf_context* ctx, int rows, int cols, const double* L, long long ldl,
                     double* B, long long ldb);
hdbf_status trsm_llu(hdbf_context* ctx, int rows, int cols, const double* L, long long ldl,
                     double* B, long long ldb);
hdbf_status syrk_lower(hdbf_context* ctx, int n, int k, const double* A, long long lda,
                       double* C, long long ldc);
hdbf_status potrf_diag(hdbf_context* ctx, int n, double* A, long long lda, int* info,
                       int info_base);
hdbf_status apply_moves(hdbf_context* ctx, double* A, long long lda, int ncols, const int* src,
                        const int* tgt, const int* count, int max_moves, double* temp,
                        long long temp_cols);
hdbf_status getrf_panel(hdbf_context* ctx, int m, int w, double* A, long long lda, int* ipiv,
                        int ipiv_add, int* info, int info_base, bool pivot, const GetrfWs& ws);
size_t getf2_coop64_scratch_bytes();
void configure_fp64_kernels(hdbf_context* ctx);
// Workspace order for a problem of order n in scalar type T: FP64 needs the
// FP32 layout of twice as many whole 64-row blocks (the inverse-block table
// holds 4096 doubles per block).
template <class T>
inline int ws_order(int n) { return sizeof(T) == 8 ? 2 * ((n + 63) / 64 * 64) : n; }
// Graph-cache key tag separating the FP32 and FP64 drivers.
template <class T>
inline long long type_tag() { return sizeof(T) == 8 ? 1000 : 0; }

// ---------------------------------------------------------------- graphs
// A whole factorization is a long chain of dependent launches; replaying it
// as one CUDA graph removes the per-launch host cost.  The first call with a
// given key records the work on a private capture stream; later calls with
// the same key replay the instantiated graph on the caller's stream.  The
// workspace must already be reserved (no allocation may happen inside).
GraphEntry* graph_find(hdbf_context* ctx, const std::vector<long long>& key);
bool graph_can_capture(hdbf_context* ctx);
hdbf_status graph_capture_begin(hdbf_context* ctx, cudaStream_t* saved);
hdbf_status graph_capture_end(hdbf_context* ctx, cudaStream_t saved, hdbf_status body_status,
                              const std::vector<long long>& key, size_t prof_mark,
                              unsigned long long launches_before);
hdbf_status graph_launch(hdbf_context* ctx, GraphEntry* e);
void graph_cache_clear(hdbf_context* ctx);

template <class Body>
hdbf_status run_graph(hdbf_context* ctx, std::vector<long long> key, Body&& body)
{
    if (!graph_can_capture(ctx)) return body();
    key.push_back(ctx->profiling ? 1 : 0);
    if (GraphEntry* e = graph_find(ctx, key)) return graph_launch(ctx, e);
    cudaStream_t saved = nullptr;
    const size_t mark = ctx->prof.size();
    const unsigned long long l0 = ctx->launches;
    if (graph_capture_begin(ctx, &saved) != HDBF_STATUS_SUCCESS) return body();
    const hdbf_status st = body();
    const hdbf_status ge = graph_capture_end(ctx, saved, st, key, mark, l0);
    if (ge == HDBF_STATUS_NOT_SUPPORTED) return body();  // capture refused: run eagerly
    return ge;
}

}  // namespace hdbf

#define HDBF_TRY(expr)                                   \
    do {                                                 \
        hdbf_status _st = (expr);                        \
        if (_st != HDBF_STATUS_SUCCESS) return _st;      \
    } while (0)
