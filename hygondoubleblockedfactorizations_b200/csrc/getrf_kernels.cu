// GETRF panel, pivot composition and row-permutation kernels (FP32).
//
// getf2_coop replaces rocsolver_sgetrf's unblocked leaf on the tall panel
// (src/getrf/getrf_pivot_internal.h:17-39): one cooperative launch factors an
// m x w (w <= 128) column block with partial pivoting.  Each CTA keeps a
// contiguous slice of rows of the block resident in shared memory; per column
// the CTAs publish their local |max| candidate (value, row and the full
// candidate row) and the owner of the diagonal row publishes that row, then
// exchange them through global memory (see the protocol note below), after
// which every CTA picks the same global winner (largest |a|, lowest row on ties -- LAPACK ISAMAX), swaps,
// scales by the reciprocal pivot (division when |pivot| < FLT_MIN, as
// xGETF2) and applies the rank-1 update to its own rows.
//
// compose_swaps + apply_moves replace apply_panel_pivots_kernel
// (src/getrf/getrf_pivot_kernels.hip:14-45) and the host-side permutation
// batching (src/getrf/getrf_batched_pivot_internal.h:59-223): a LAPACK swap
// sequence is composed on the GPU into a list of (source, target) row moves,
// then applied to column tiles with a gather into shared memory followed by a
// scatter -- no host round trip.
#include <cfloat>
#include <climits>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int kCoopThreads = 256;
constexpr int kCoopMaxW = 128;
constexpr int kCoopMaxGrid = 256;
// Per-(parity, CTA) exchange slot: [seq, |val|, row, pad | cand row (32) | diag row (32)]
constexpr int kSlotFloats = 4 + 2 * kCoopMaxW;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Candidate (v, i) beats (bv, bi): a real row beats none, then larger |a|,
// then the lower row (LAPACK ISAMAX returns the first maximum).
__device__ __forceinline__ bool better(float v, int i, float bv, int bi)
{
    if (i == INT_MAX) return false;
    if (bi == INT_MAX) return true;
    return v > bv || (v == bv && i < bi);
}

// Copy an nr x w column block between global memory and the shared tile
// (leading dimension ldt), eight independent loads in flight per thread.
template <bool TO_SMEM>
__device__ __forceinline__ void coop_move(float* A, long long lda, float* tile, int ldt, int nr,
                                          int w)
{
    const int total = nr * w;
    int e = threadIdx.x;
    for (; e + 7 * kCoopThreads < total; e += 8 * kCoopThreads) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kCoopThreads, c = q / nr, r = q - c * nr;
            v[u] = TO_SMEM ? A[(long long)c * lda + r] : tile[c * ldt + r];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kCoopThreads, c = q / nr, r = q - c * nr;
            if (TO_SMEM) tile[c * ldt + r] = v[u];
            else A[(long long)c * lda + r] = v[u];
        }
    }
    for (; e < total; e += kCoopThreads) {
        const int c = e / nr, r = e - c * nr;
        if (TO_SMEM) tile[c * ldt + r] = A[(long long)c * lda + r];
        else A[(long long)c * lda + r] = tile[c * ldt + r];
    }
}

// Exchange protocol (no grid barrier): for column j every CTA writes its slot
// (parity j&1) -- candidate |max|, its row index and that row's w values, plus
// the diagonal row j if it owns it -- then publishes seq = epoch*64 + j + 1
// with a release store.  Every CTA polls all G seq words with acquire loads
// (bounded), reduces the candidates identically, and fetches the winning row
// and the old diagonal row.  A CTA can only overwrite a parity slot after all
// CTAs have published the following column, i.e. after every CTA finished
// reading that slot, so two parities suffice.  `epoch` is read at entry and
// advanced by the last CTA to finish, so slots of earlier launches (and of
// earlier CUDA-graph replays) never match.
__global__ void __launch_bounds__(kCoopThreads)
getf2_coop_kernel(int m, int w, float* A, long long lda, int rpc, int* ipiv, int ipiv_add,
                  int* info, int info_base, float* scr, unsigned* epoch_ptr, unsigned* done_ptr,
                  int* err, int pivot)
{
    extern __shared__ float tile[];  // tile[c * rpc + r]
    __shared__ float prow[kCoopMaxW];
    __shared__ float orow[kCoopMaxW];
    __shared__ float red_v[kCoopThreads / 32];
    __shared__ int red_i[kCoopThreads / 32];
    __shared__ float cv[kCoopMaxGrid];
    __shared__ int ci[kCoopMaxGrid];
    __shared__ int s_best_row, s_win_cta, s_abort;

    const int G = gridDim.x;
    const int cta = blockIdx.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int r0 = cta * rpc;
    const int nr = max(0, min(m, r0 + rpc) - r0);
    const unsigned epoch = *reinterpret_cast<volatile unsigned*>(epoch_ptr);

    coop_move<true>(A + r0, lda, tile, rpc, nr, w);
    if (tid == 0) s_abort = 0;
    __syncthreads();

    const int steps = min(m, w);
    for (int j = 0; j < steps; ++j) {
        const int par = j & 1;
        const unsigned seq = (epoch << 6) + (unsigned)j + 1u;
        float* slot = scr + ((long long)par * kCoopMaxGrid + cta) * kSlotFloats;
        const int owner = j / rpc;

        // 1. local candidate over owned rows >= j (largest |a|, lowest row)
        float bv = -1.f;
        int bi = INT_MAX;
        if (pivot) {
            for (int r = tid; r < nr; r += kCoopThreads) {
                const int gr = r0 + r;
                if (gr >= j) {
                    const float v = fabsf(tile[j * rpc + r]);
                    if (bi == INT_MAX || v > bv) { bv = v; bi = gr; }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float ov = __shfl_down_sync(0xffffffffu, bv, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
            }
            if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
            __syncthreads();
            if (tid == 0) {
                for (int q = 1; q < kCoopThreads / 32; ++q)
                    if (better(red_v[q], red_i[q], bv, bi)) { bv = red_v[q]; bi = red_i[q]; }
                s_best_row = bi;
                red_v[0] = bv;
            }
            __syncthreads();
        }

        // 2. publish
        const int my_best = pivot ? s_best_row : INT_MAX;
        if (tid < w) {
            if (my_best != INT_MAX) slot[4 + tid] = tile[tid * rpc + (my_best - r0)];
            if (cta == owner) slot[4 + kCoopMaxW + tid] = tile[tid * rpc + (j - r0)];
        }
        if (tid == 0) {
            slot[1] = pivot ? red_v[0] : -1.f;
            slot[2] = __int_as_float(my_best);
        }
        __syncthreads();
        // The release store (after the barrier) orders every thread's slot
        // writes before the sequence number that other CTAs acquire.
        if (tid == 0) st_release_u32(reinterpret_cast<unsigned*>(slot), seq);

        // 3. poll every slot (thread q watches CTA q), bounded
        for (int q = tid; q < G; q += kCoopThreads) {
            const float* sq = scr + ((long long)par * kCoopMaxGrid + q) * kSlotFloats;
            unsigned polls = 0;
            while (ld_acquire_u32(reinterpret_cast<const unsigned*>(sq)) != seq) {
                if (++polls > kSpinLimit) {
                    atomicExch(err, kErrTimeout);
                    s_abort = 1;
                    break;
                }
                if (polls > 256) __nanosleep(32);
            }
            cv[q] = __ldcg(sq + 1);
            ci[q] = __float_as_int(__ldcg(sq + 2));
        }
        __syncthreads();
        if (s_abort) break;

        // 4. global winner, identical on every CTA
        if (!pivot) {
            if (tid == 0) { s_best_row = j; s_win_cta = -1; }
        } else if (warp == 0) {
            float gv = -1.f;
            int gi = INT_MAX, gc = 0;
            for (int q = lane; q < G; q += 32)
                if (better(cv[q], ci[q], gv, gi)) { gv = cv[q]; gi = ci[q]; gc = q; }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float ov = __shfl_down_sync(0xffffffffu, gv, off);
                const int oi = __shfl_down_sync(0xffffffffu, gi, off);
                const int oc = __shfl_down_sync(0xffffffffu, gc, off);
                if (better(ov, oi, gv, gi)) { gv = ov; gi = oi; gc = oc; }
            }
            if (lane == 0) { s_best_row = gi; s_win_cta = gc; }
        }
        __syncthreads();
        const int p = s_best_row;
        if (tid < w) {
            const float* so = scr + ((long long)par * kCoopMaxGrid + owner) * kSlotFloats;
            orow[tid] = __ldcg(so + 4 + kCoopMaxW + tid);
            if (s_win_cta >= 0) {
                const float* sw = scr + ((long long)par * kCoopMaxGrid + s_win_cta) * kSlotFloats;
                prow[tid] = __ldcg(sw + 4 + tid);
            } else {
                prow[tid] = orow[tid];
            }
        }
        if (pivot && cta == 0 && tid == 0) ipiv[j] = p + 1 + ipiv_add;
        __syncthreads();

        // 5. swap rows j and p (within this column block), scale, rank-1 update
        if (p != j && tid < w) {
            if (j >= r0 && j < r0 + nr) tile[tid * rpc + (j - r0)] = prow[tid];
            if (p >= r0 && p < r0 + nr) tile[tid * rpc + (p - r0)] = orow[tid];
        }
        __syncthreads();
        const float piv = prow[j];
        const bool nz = piv != 0.f;
        const bool recip = fabsf(piv) >= FLT_MIN;
        const float rcp = 1.0f / piv;
        if (!nz && cta == 0 && tid == 0 && info) atomicCAS(info, 0, info_base + j + 1);
        for (int r = tid; r < nr; r += kCoopThreads) {
            if (r0 + r > j) {
                float l = tile[j * rpc + r];
                if (nz) {
                    l = recip ? l * rcp : l / piv;
                    tile[j * rpc + r] = l;
                }
                for (int c = j + 1; c < w; ++c) tile[c * rpc + r] = fmaf(-l, prow[c], tile[c * rpc + r]);
            }
        }
        __syncthreads();
    }

    coop_move<false>(A + r0, lda, tile, rpc, nr, w);

    // Advance the epoch once every CTA is done (the kernel's last action).
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        const unsigned done = atomicAdd(done_ptr, 1u) + 1u;
        if (done == (unsigned)G) {
            atomicExch(done_ptr, 0u);
            atomicAdd(epoch_ptr, 1u);
        }
    }
}

// ------------------------------------------------------------ compose swaps
constexpr int kComposeThreads = 1024;

__global__ void __launch_bounds__(kComposeThreads)
compose_swaps_kernel(const int* __restrict__ ipiv, int k, int ipiv_minus, int m, int* src,
                     int* tgt, int* count, int* gperm, int use_smem, int* info, int* err)
{
    // Shared layout (use_smem): perm[m] then the k pivots; otherwise perm
    // lives in global scratch and the pivots are re-read from global memory.
    extern __shared__ int sperm[];
    __shared__ int warp_tot[kComposeThreads / 32];
    __shared__ int s_base, s_bad, s_chunk;
    int* perm = use_smem ? sperm : gperm;
    int* piv = use_smem ? sperm + m : nullptr;
    const int tid = threadIdx.x;
    if (tid == 0) { s_bad = 0; s_base = 0; }
    __syncthreads();
    for (int q = tid; q < m; q += kComposeThreads) perm[q] = q;
    for (int i = tid; i < k; i += kComposeThreads) {
        const int b = ipiv[i] - 1 - ipiv_minus;
        if (b < i || b >= m) s_bad = 1;
        if (piv) piv[i] = b;
    }
    __syncthreads();
    if (s_bad) {
        if (tid == 0) {
            *count = 0;
            if (info) atomicExch(info, -1);
            atomicExch(err, kErrBadPivot);
        }
        return;
    }
    // The swap sequence itself is inherently ordered: one thread replays it.
    if (tid == 0) {
        for (int i = 0; i < k; ++i) {
            const int b = piv ? piv[i] : ipiv[i] - 1 - ipiv_minus;
            if (b != i) {
                const int t = perm[i];
                perm[i] = perm[b];
                perm[b] = t;
            }
        }
    }
    __syncthreads();
    // Moves: rows [0, k) in order (ordered block scan), then the distinct
    // pivot rows >= k (each claimed once by flipping its entry negative).
    const int lane = tid & 31, warp = tid >> 5;
    for (int q0 = 0; q0 < k; q0 += kComposeThreads) {
        const int q = q0 + tid;
        const int s = (q < k) ? perm[q] : q;
        const bool moved = (q < k) && (s != q);
        const unsigned ball = __ballot_sync(0xffffffffu, moved);
        const int within = __popc(ball & ((1u << lane) - 1u));
        if (lane == 0) warp_tot[warp] = __popc(ball);
        __syncthreads();
        if (tid == 0) {
            int run = 0;
            for (int wv = 0; wv < kComposeThreads / 32; ++wv) {
                const int t = warp_tot[wv];
                warp_tot[wv] = run;
                run += t;
            }
            s_chunk = run;
        }
        __syncthreads();
        if (moved) {
            const int pos = s_base + warp_tot[warp] + within;
            src[pos] = s;
            tgt[pos] = q;
        }
        __syncthreads();
        if (tid == 0) s_base += s_chunk;
        __syncthreads();
    }
    for (int i = tid; i < k; i += kComposeThreads) {
        const int b = piv ? piv[i] : ipiv[i] - 1 - ipiv_minus;
        if (b < k) continue;
        const int s = atomicExch(&perm[b], -1);  // claim position b once
        if (s >= 0 && s != b) {
            const int pos = atomicAdd(&s_base, 1);
            src[pos] = s;
            tgt[pos] = b;
        }
    }
    __syncthreads();
    if (tid == 0) *count = s_base;
}

// ------------------------------------------------------------ apply moves
constexpr int kApplyThreads = 256;

// Columns [blockIdx.x*cpc, +cpc): gather every source row into shared memory,
// then scatter to the targets.  Sources and targets are the same row set, so
// reading everything before writing anything is race-free per column.
__global__ void __launch_bounds__(kApplyThreads)
apply_moves_smem_kernel(float* A, long long lda, int ncols, const int* __restrict__ src,
                        const int* __restrict__ tgt, const int* __restrict__ count, int cpc,
                        int cap)
{
    extern __shared__ float buf[];  // cpc * cap values, then cap sources, cap targets
    int* s_src = reinterpret_cast<int*>(buf + (size_t)cpc * cap);
    int* s_tgt = s_src + cap;
    const int cnt = min(*count, cap);
    if (cnt <= 0) return;
    const int c0 = blockIdx.x * cpc;
    const int nc = min(cpc, ncols - c0);
    for (int i = threadIdx.x; i < cnt; i += kApplyThreads) {
        s_src[i] = src[i];
        s_tgt[i] = tgt[i];
    }
    __syncthreads();
    // Flattened (column, move) space, eight independent loads in flight.
    const int total = nc * cnt;
    const float* base = A + (long long)c0 * lda;
    int e = threadIdx.x;
    for (; e + 7 * kApplyThreads < total; e += 8 * kApplyThreads) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kApplyThreads, cc = q / cnt, i = q - cc * cnt;
            v[u] = base[(long long)cc * lda + s_src[i]];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kApplyThreads, cc = q / cnt, i = q - cc * cnt;
            buf[cc * cap + i] = v[u];
        }
    }
    for (; e < total; e += kApplyThreads) {
        const int cc = e / cnt, i = e - cc * cnt;
        buf[cc * cap + i] = base[(long long)cc * lda + s_src[i]];
    }
    __syncthreads();
    float* wbase = A + (long long)c0 * lda;
    for (int q = threadIdx.x; q < total; q += kApplyThreads) {
        const int cc = q / cnt, i = q - cc * cnt;
        wbase[(long long)cc * lda + s_tgt[i]] = buf[cc * cap + i];
    }
}

__global__ void gather_rows_kernel(const float* A, long long lda, int ncols,
                                   const int* __restrict__ src, const int* __restrict__ count,
                                   int cap, float* temp)
{
    const int cnt = min(*count, cap);
    const long long total = (long long)cnt * ncols;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % cnt);
        const long long c = idx / cnt;
        temp[c * cap + i] = A[c * lda + src[i]];
    }
}

__global__ void scatter_rows_kernel(float* A, long long lda, int ncols,
                                    const int* __restrict__ tgt, const int* __restrict__ count,
                                    int cap, const float* temp)
{
    const int cnt = min(*count, cap);
    const long long total = (long long)cnt * ncols;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx % cnt);
        const long long c = idx / cnt;
        A[c * lda + tgt[i]] = temp[c * cap + i];
    }
}

}  // namespace

// Dynamic shared-memory opt-ins, set once per handle creation (never inside a
// stream capture).
void configure_getrf_kernels(hdbf_context* ctx)
{
    const size_t cap8 = ctx->max_smem_optin > 8192 ? ctx->max_smem_optin - 8192 : 40960;
    const size_t cap4 = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    cudaFuncSetAttribute(getf2_coop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap8);
    cudaFuncSetAttribute(compose_swaps_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap4);
    cudaFuncSetAttribute(apply_moves_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap4);
    cudaGetLastError();
}

size_t getf2_coop_scratch_bytes()
{
    return align_up((size_t)(2 * kCoopMaxGrid * kSlotFloats) * sizeof(float), 256);
}

hdbf_status getf2_coop(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                       int ipiv_add, int* info, int info_base, bool pivot)
{
    int piv_flag = pivot ? 1 : 0;
    if (m <= 0 || w <= 0) return HDBF_STATUS_SUCCESS;
    if (w > kCoopMaxW) return HDBF_STATUS_INVALID_VALUE;
    HDBF_TRY(ensure_ws(ctx, 64));
    float* scr = ws_coop(ctx);

    // Grid: ~256 rows per CTA (panel_rows; measured fastest at n = 32768),
    // more when the slice would not fit in shared memory, at most one CTA per
    // SM; co-residency is guaranteed by the cooperative launch, which fails
    // instead of hanging if the grid cannot fit.
    const size_t smem_cap = ctx->max_smem_optin > 8192 ? ctx->max_smem_optin - 8192 : 40960;
    const size_t row_bytes = (size_t)w * sizeof(float);
    const long long fit_rows = (long long)(smem_cap / row_bytes);
    const int target = ctx->panel_rows > 0 ? ctx->panel_rows : 256;
    int G = (m + target - 1) / target;
    if (fit_rows > 0 && (m + fit_rows - 1) / fit_rows > G) G = (int)((m + fit_rows - 1) / fit_rows);
    if (G > ctx->sm_count) G = ctx->sm_count;
    if (G > kCoopMaxGrid) G = kCoopMaxGrid;
    if (G < 1) G = 1;
    int rpc = (m + G - 1) / G;
    size_t smem = (size_t)rpc * w * sizeof(float);
    if (smem > smem_cap) return HDBF_STATUS_NOT_SUPPORTED;
    unsigned* epoch = reinterpret_cast<unsigned*>(ctx->dev_small + kSmallEpoch);
    unsigned* done = reinterpret_cast<unsigned*>(ctx->dev_small + kSmallDone);
    int* err = ctx->dev_small + kSmallErr;
    ProfScope prof(ctx, kClsPanel, (double)m * w * w - (double)w * w * w / 3.0, 8.0 * m * w);
    void* args[] = {&m, &w, &A, &lda, &rpc, &ipiv, &ipiv_add, &info, &info_base,
                    &scr, &epoch, &done, &err, &piv_flag};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)getf2_coop_kernel, dim3(G),
                                                dim3(kCoopThreads), args, smem, ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    return HDBF_STATUS_SUCCESS;
}

hdbf_status compose_swaps(hdbf_context* ctx, const int* ipiv, int k, int ipiv_minus, int m,
                          int* src, int* tgt, int* count, int* gperm, int* info)
{
    if (k <= 0 || m <= 0) return HDBF_STATUS_SUCCESS;
    const size_t smem = ((size_t)m + (size_t)k) * sizeof(int);
    const size_t cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    const int use_smem = smem <= cap ? 1 : 0;
    if (!use_smem && !gperm) return HDBF_STATUS_INVALID_VALUE;
    ProfScope prof(ctx, kClsCompose, 0.0, 4.0 * k + 8.0 * m);
    compose_swaps_kernel<<<1, kComposeThreads, use_smem ? smem : 0, ctx->stream>>>(
        ipiv, k, ipiv_minus, m, src, tgt, count, gperm, use_smem, info,
        ctx->dev_small + kSmallErr);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status apply_moves(hdbf_context* ctx, float* A, long long lda, int ncols,
                        const int* src, const int* tgt, const int* count, int max_moves,
                        float* temp, long long temp_cols)
{
    if (ncols <= 0 || max_moves <= 0) return HDBF_STATUS_SUCCESS;
    const size_t per_col = (size_t)max_moves * sizeof(float);
    const size_t idx_bytes = 2 * (size_t)max_moves * sizeof(int);
    const size_t budget = 64 * 1024;
    const size_t hard_cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    ProfScope prof(ctx, kClsMoves, 0.0, 8.0 * (double)max_moves * ncols);
    if (per_col + idx_bytes <= hard_cap) {
        int cpc = (int)((budget > idx_bytes ? budget - idx_bytes : 0) / per_col);
        if (cpc < 1) cpc = 1;
        if (cpc > 16) cpc = 16;
        const int grid = (ncols + cpc - 1) / cpc;
        apply_moves_smem_kernel<<<grid, kApplyThreads, per_col * cpc + idx_bytes, ctx->stream>>>(
            A, lda, ncols, src, tgt, count, cpc, max_moves);
        ctx->launches++;
        return last_cuda(ctx);
    }
    if (!temp || temp_cols <= 0) return HDBF_STATUS_INVALID_VALUE;
    for (long long c = 0; c < ncols; c += temp_cols) {
        const int nc = (int)((ncols - c) < temp_cols ? (ncols - c) : temp_cols);
        const long long total = (long long)nc * max_moves;
        const int grid = (int)((total + 255) / 256 < 65535 ? (total + 255) / 256 : 65535);
        gather_rows_kernel<<<grid, 256, 0, ctx->stream>>>(A + c * lda, lda, nc, src, count,
                                                          max_moves, temp);
        scatter_rows_kernel<<<grid, 256, 0, ctx->stream>>>(A + c * lda, lda, nc, tgt, count,
                                                           max_moves, temp);
        ctx->launches += 2;
    }
    return last_cuda(ctx);
}

}  // namespace hdbf
