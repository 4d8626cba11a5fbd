// GETRF panel leaf on one thread-block cluster: partially pivoted LU of an
// m x w (w <= 32) column block, replacing rocsolver_sgetrf's unblocked leaf on
// the tall panel (src/getrf/getrf_pivot_internal.h:17-39) whenever the block
// fits in the shared memory of one cluster (up to 16 CTAs).
//
// Each CTA of the cluster keeps a contiguous slice of rows resident in shared
// memory (column-major tile[c * ldt + r], ldt = rpc rounded up to odd); thread t
// owns local rows t, t + T,
// ...  Per column j:
//   1. every CTA finds its candidate (largest |a| over owned rows >= j, lowest
//      row on ties -- LAPACK ISAMAX) and writes it, the candidate row and (on
//      the CTA owning row j) the diagonal row into its own slot (two parities);
//   2. one cluster barrier (release / acquire);
//   3. warp 0 of every CTA reads the cluster's candidates through distributed
//      shared memory, reduces them identically, and copies the winning row and
//      the diagonal row from their slots (copies, so owners may overwrite their
//      live rows at once) into local shared memory for the other warps;
//   4. the owners swap rows j and p, every thread scales its rows below j by
//      the reciprocal pivot (division when |pivot| < FLT_MIN, as xGETF2) and
//      applies the rank-1 update to its own rows.
// A slot of parity j & 1 is rewritten at column j + 2 only after the barrier
// of column j + 1, which every CTA reaches after its reads of column j, so two
// parities suffice.  All CTAs run the same loop, so every cluster barrier is
// met; there are no spin-waits.
#include <cfloat>
#include <climits>
#include <cooperative_groups.h>

#include "internal.h"

namespace cg = cooperative_groups;

namespace hdbf {
namespace {

constexpr int kClThreads = 256;
constexpr int kClMaxW = 32;
constexpr int kClSlot = 4 + 2 * kClMaxW;  // [|v|, row, -, - | candidate row | diagonal row]
constexpr int kClMaxCluster = 16;

__device__ __forceinline__ bool better(float v, int i, float bv, int bi)
{
    if (i == INT_MAX) return false;
    if (bi == INT_MAX) return true;
    return v > bv || (v == bv && i < bi);
}

// Copy an nr x w column block between global memory (leading dimension lda)
// and the shared tile (leading dimension ldt), eight independent loads in
// flight per thread.
template <bool TO_SMEM>
__device__ __forceinline__ void move_block(float* A, long long lda, float* tile, int ldt, int nr,
                                           int w)
{
    const int total = nr * w;
    int e = threadIdx.x;
    for (; e + 7 * kClThreads < total; e += 8 * kClThreads) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kClThreads, c = q / nr, r = q - c * nr;
            v[u] = TO_SMEM ? A[(long long)c * lda + r] : tile[c * ldt + r];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * kClThreads, c = q / nr, r = q - c * nr;
            if (TO_SMEM) tile[c * ldt + r] = v[u];
            else A[(long long)c * lda + r] = v[u];
        }
    }
    for (; e < total; e += kClThreads) {
        const int c = e / nr, r = e - c * nr;
        if (TO_SMEM) tile[c * ldt + r] = A[(long long)c * lda + r];
        else A[(long long)c * lda + r] = tile[c * ldt + r];
    }
}

__global__ void __launch_bounds__(kClThreads, 1)
getf2_cluster_kernel(int m, int w, float* A, long long lda, int rpc, int ldt, int* ipiv,
                     int ipiv_add, int* info, int info_base, int pivot)
{
    extern __shared__ __align__(16) float smem[];
    float* slots = smem;               // [2][kClSlot]
    float* tile = smem + 2 * kClSlot;  // tile[c * ldt + r], ldt odd (no bank conflicts)
    __shared__ float red_v[kClThreads / 32];
    __shared__ int red_i[kClThreads / 32];
    __shared__ float s_prow[kClMaxW], s_orow[kClMaxW];
    __shared__ int s_p;

    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = rank * rpc;
    const int nr = max(0, min(m, r0 + rpc) - r0);

    move_block<true>(A + r0, lda, tile, ldt, nr, w);
    cluster.sync();  // every CTA of the cluster is running before any DSMEM access

    const int steps = min(m, w);
    for (int j = 0; j < steps; ++j) {
        const int par = j & 1;
        float* my_slot = slots + par * kClSlot;
        const int owner = j / rpc;

        // 1. local candidate
        float bv = -1.f;
        int bi = INT_MAX;
        if (pivot) {
            for (int r = tid; r < nr; r += kClThreads) {
                if (r0 + r >= j) {
                    const float v = fabsf(tile[j * ldt + r]);
                    if (bi == INT_MAX || v > bv) { bv = v; bi = r0 + r; }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float ov = __shfl_down_sync(0xffffffffu, bv, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
            }
            if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
        }
        __syncthreads();
        if (warp == 0) {
            if (pivot) {
                bv = lane < kClThreads / 32 ? red_v[lane] : -1.f;
                bi = lane < kClThreads / 32 ? red_i[lane] : INT_MAX;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const float ov = __shfl_down_sync(0xffffffffu, bv, off);
                    const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                    if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
                }
                bv = __shfl_sync(0xffffffffu, bv, 0);
                bi = __shfl_sync(0xffffffffu, bi, 0);
            }
            if (lane == 0) {
                my_slot[0] = bv;
                my_slot[1] = __int_as_float(bi);
            }
            if (lane < w) {
                if (bi != INT_MAX) my_slot[4 + lane] = tile[lane * ldt + (bi - r0)];
                if (rank == owner) my_slot[4 + kClMaxW + lane] = tile[lane * ldt + (j - r0)];
            }
        }
        // 2. publish to the cluster
        cluster.sync();

        // 3. warp 0 gathers the cluster's candidates and the two rows
        if (warp == 0) {
            float gv = -1.f;
            int gi = INT_MAX, gc = -1;
            if (pivot) {
                if (lane < C) {
                    const float* rs = cluster.map_shared_rank(slots, lane) + par * kClSlot;
                    gv = rs[0];
                    gi = __float_as_int(rs[1]);
                    gc = lane;
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const float ov = __shfl_down_sync(0xffffffffu, gv, off);
                    const int oi = __shfl_down_sync(0xffffffffu, gi, off);
                    const int oc = __shfl_down_sync(0xffffffffu, gc, off);
                    if (better(ov, oi, gv, gi)) { gv = ov; gi = oi; gc = oc; }
                }
                gi = __shfl_sync(0xffffffffu, gi, 0);
                gc = __shfl_sync(0xffffffffu, gc, 0);
            }
            if (lane < w) {
                const float* os = cluster.map_shared_rank(slots, owner) + par * kClSlot;
                const float ov = os[4 + kClMaxW + lane];
                s_orow[lane] = ov;
                if (pivot) {
                    const float* ws = cluster.map_shared_rank(slots, gc) + par * kClSlot;
                    s_prow[lane] = ws[4 + lane];
                } else {
                    s_prow[lane] = ov;
                }
            }
            if (lane == 0) {
                s_p = pivot ? gi : j;
                if (pivot && rank == 0) ipiv[j] = (pivot ? gi : j) + 1 + ipiv_add;
            }
        }
        __syncthreads();

        // 4. swap, scale, rank-1 update (each thread on its own rows)
        const int p = s_p;
        const float piv = s_prow[j];
        const bool nz = piv != 0.f;
        const bool recip = fabsf(piv) >= FLT_MIN;
        const float rcp = 1.0f / piv;
        if (!nz && rank == 0 && tid == 0 && info) atomicCAS(info, 0, info_base + j + 1);
        if (j >= r0 && j < r0 + nr && ((j - r0) % kClThreads) == tid)
            for (int c = 0; c < w; ++c) tile[c * ldt + (j - r0)] = s_prow[c];
        if (p != j && p >= r0 && p < r0 + nr && ((p - r0) % kClThreads) == tid)
            for (int c = 0; c < w; ++c) tile[c * ldt + (p - r0)] = s_orow[c];
        for (int r = tid; r < nr; r += kClThreads) {
            if (r0 + r > j) {
                float l = tile[j * ldt + r];
                if (nz) {
                    l = recip ? l * rcp : l / piv;
                    tile[j * ldt + r] = l;
                }
                for (int c = j + 1; c < w; ++c)
                    tile[c * ldt + r] = fmaf(-l, s_prow[c], tile[c * ldt + r]);
            }
        }
    }
    __syncthreads();
    move_block<false>(A + r0, lda, tile, ldt, nr, w);
    cluster.sync();  // no CTA leaves while another may still read its slots
}

int cluster_ldt(int rpc) { return rpc | 1; }
size_t cluster_smem(int rpc, int w)
{
    return sizeof(float) * (2 * (size_t)kClSlot + (size_t)cluster_ldt(rpc) * w);
}

}  // namespace

int configure_cluster_panel(hdbf_context* ctx)
{
    const size_t cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    cudaFuncSetAttribute(getf2_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
    cudaFuncSetAttribute(getf2_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaGetLastError();
    int best = 0;
    for (int C = kClMaxCluster; C >= 1 && best == 0; C /= 2) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(kClThreads);
        cfg.dynamicSmemBytes = cap;
        cudaLaunchAttribute at;
        at.id = cudaLaunchAttributeClusterDimension;
        at.val.clusterDim.x = C;
        at.val.clusterDim.y = 1;
        at.val.clusterDim.z = 1;
        cfg.attrs = &at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, getf2_cluster_kernel, &cfg) == cudaSuccess &&
            clusters >= 1)
            best = C;
        cudaGetLastError();
    }
    return best;
}

hdbf_status getf2_cluster(hdbf_context* ctx, int m, int w, float* A, long long lda, int* ipiv,
                          int ipiv_add, int* info, int info_base, bool pivot)
{
    if (m <= 0 || w <= 0) return HDBF_STATUS_SUCCESS;
    if (w > kClMaxW || ctx->cluster_max < 1) return HDBF_STATUS_NOT_SUPPORTED;
    const size_t cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    // Fewest CTAs whose slices fit, but at most 8 rows per thread.
    int C = 1;
    while (C < ctx->cluster_max &&
           (cluster_smem((m + C - 1) / C, w) > cap || (m + C - 1) / C > 8 * kClThreads))
        C *= 2;
    const int rpc = (m + C - 1) / C;
    const int ldt = cluster_ldt(rpc);
    const size_t smem = cluster_smem(rpc, w);
    if (smem > cap) return HDBF_STATUS_NOT_SUPPORTED;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = C;
    at.val.clusterDim.y = 1;
    at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    const int piv_flag = pivot ? 1 : 0;
    ProfScope prof(ctx, kClsPanel, (double)m * w * w - (double)w * w * w / 3.0, 8.0 * m * w);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, getf2_cluster_kernel, m, w, A, lda, rpc, ldt,
                                             ipiv, ipiv_add, info, info_base, piv_flag);
    ctx->launches++;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    return HDBF_STATUS_SUCCESS;
}

}  // namespace hdbf
