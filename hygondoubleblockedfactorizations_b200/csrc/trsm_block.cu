// Coarse leaves of the recursive TRSMs: left/lower/unit B <- L^{-1} B
// (rows <= 256) and right/lower/transposed B <- B L^{-T} (cols <= 256).
//
// The recursive TRSM (trsm_llu in drivers.cu, replacing the reference's
// trsm_left_lower_unit, src/getrf/getrf_npvt_internal.h:42-88) used to
// recurse down to 64-row leaves, which produced GEMMs with M = K = 64 -- each a
// latency-bound launch.  This kernel solves up to four 64-row blocks at once:
// a CTA keeps 64 columns of B (all rows) in shared memory and runs the block
// forward substitution
//     X_i = D_i (B_i - sum_{j<i} L_ij X_j),   D_i = L_ii^{-1}
// with 64 x 64 tile products (D_i from tri_inv64, unit diagonal).
#include "internal.h"

namespace hdbf {
namespace {

constexpr int kT = 64;
constexpr int kThreads = 256;
constexpr int kMaxRows = 256;
constexpr int kLdS = 68;

__device__ __forceinline__ void tile_mma(float acc[4][4], const float* As, const float* Bs)
{
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll 8
    for (int k = 0; k < kT; ++k) {
        const float4 a = *reinterpret_cast<const float4*>(As + k * kLdS + ty * 4);
        const float4 b = *reinterpret_cast<const float4*>(Bs + k * kLdS + tx * 4);
        const float av[4] = {a.x, a.y, a.z, a.w};
        const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
}

// As[k][m] = src(m, k) = src[k * ld + m] for m < rows, k < cols (else 0)
__device__ __forceinline__ void load_kmajor(float* As, const float* src, long long ld, int rows,
                                            int cols)
{
    for (int q = threadIdx.x; q < kT * kT; q += kThreads) {
        const int k = q >> 6, m = q & 63;
        As[k * kLdS + m] = (m < rows && k < cols) ? src[(long long)k * ld + m] : 0.f;
    }
}

// 64 x 64 tile into shared memory, k-major (As[k][m] = src(m, k) =
// src[k * ld + m], zero outside rows x cols), every load of the thread in
// flight before the first store.
__device__ __forceinline__ void load_kmajor_batched(float* As, const float* src, long long ld,
                                                    int rows, int cols)
{
    float v[kT * kT / kThreads];
#pragma unroll
    for (int u = 0; u < kT * kT / kThreads; ++u) {
        const int q = threadIdx.x + u * kThreads, k = q >> 6, m = q & 63;
        v[u] = (m < rows && k < cols) ? src[(long long)k * ld + m] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kT * kT / kThreads; ++u) {
        const int q = threadIdx.x + u * kThreads, k = q >> 6, m = q & 63;
        As[k * kLdS + m] = v[u];
    }
}

// acc[a][b] += sum_k As[k][ty*4+a] * Xs[k][tx*CW+b] (64 rows x 16*CW columns)
template <int CW>
__device__ __forceinline__ void tile_mma_cw(float acc[4][CW], const float* As, const float* Xs,
                                            int ldx)
{
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll 8
    for (int k = 0; k < kT; ++k) {
        const float4 a = *reinterpret_cast<const float4*>(As + k * kLdS + ty * 4);
        const float av[4] = {a.x, a.y, a.z, a.w};
        float bv[CW];
#pragma unroll
        for (int b = 0; b < CW; ++b) bv[b] = Xs[k * ldx + tx * CW + b];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < CW; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
}

// B <- L^{-1} B for a column slice of CT = 16 * CW columns per CTA (all
// rows <= 256 in shared memory): narrow right-hand sides get more CTAs.
template <int CW>
__global__ void __launch_bounds__(kThreads) llu_block_kernel(int rows, int cols,
                                                             const float* __restrict__ L,
                                                             long long ldl,
                                                             const float* __restrict__ inv,
                                                             float* B, long long ldb)
{
    constexpr int CT = 16 * CW;
    constexpr int LDX = CT + 4;
    extern __shared__ __align__(16) float sm[];
    float* Xs = sm;                       // kMaxRows x LDX: Xs[r][c] = B(r, c0 + c)
    float* As = Xs + kMaxRows * LDX;      // left operand tile (k-major)
    float* Ts = As + kT * kLdS;           // right operand staging (64 x LDX)
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const long long c0 = (long long)blockIdx.x * CT;
    const int nc = (int)min((long long)CT, (long long)cols - c0);
    const int nb = (rows + kT - 1) / kT;

    for (int q = tid; q < kMaxRows * CT; q += kThreads) {
        const int c = q / kMaxRows, r = q - c * kMaxRows;
        Xs[r * LDX + c] = (r < rows && c < nc) ? B[(c0 + c) * ldb + r] : 0.f;
    }
    __syncthreads();
    for (int i = 0; i < nb; ++i) {
        const int ri = min(kT, rows - i * kT);
        float acc[4][CW];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < CW; ++b) acc[a][b] = Xs[(i * kT + ty * 4 + a) * LDX + tx * CW + b];
        for (int j = 0; j < i; ++j) {
            load_kmajor_batched(As, L + (long long)(j * kT) * ldl + i * kT, ldl, ri, kT);
            __syncthreads();
            float p[4][CW] = {};
            tile_mma_cw<CW>(p, As, Xs + j * kT * LDX, LDX);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < CW; ++b) acc[a][b] -= p[a][b];
            __syncthreads();
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < CW; ++b) Ts[(ty * 4 + a) * LDX + tx * CW + b] = acc[a][b];
        load_kmajor_batched(As, inv + (long long)i * kT * kT, kT, kT, kT);
        __syncthreads();
        float x[4][CW] = {};
        tile_mma_cw<CW>(x, As, Ts, LDX);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < CW; ++b)
                Xs[(i * kT + ty * 4 + a) * LDX + tx * CW + b] = (ty * 4 + a < ri) ? x[a][b] : 0.f;
        __syncthreads();
    }
    for (int q = tid; q < kMaxRows * CT; q += kThreads) {
        const int c = q / kMaxRows, r = q - c * kMaxRows;
        if (r < rows && c < nc) B[(c0 + c) * ldb + r] = Xs[r * LDX + c];
    }
}

// B(rows x cols <= 256) <- B L^{-T}, L lower non-unit: a CTA keeps 64 rows of
// B (all columns) in shared memory, column-major (Xs[c][r]), and runs
//     X_j = (B_j - sum_{i<j} X_i L_ji^T) D_j^T,   D_j = L_jj^{-1}.
__global__ void __launch_bounds__(kThreads) rlt_block_kernel(int rows, int cols,
                                                             const float* __restrict__ L,
                                                             long long ldl,
                                                             const float* __restrict__ inv,
                                                             float* B, long long ldb)
{
    extern __shared__ __align__(16) float sm[];
    float* Xs = sm;                       // kMaxRows (columns) x kLdS: Xs[c][r] = B(r0 + r, c)
    float* Bs = Xs + kMaxRows * kLdS;     // right operand tile
    float* Ts = Bs + kT * kLdS;           // left operand staging
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const long long r0 = (long long)blockIdx.x * kT;
    const int nr = (int)min((long long)kT, (long long)rows - r0);
    const int nb = (cols + kT - 1) / kT;

    for (int q = tid; q < kMaxRows * kT; q += kThreads) {
        const int c = q >> 6, r = q & 63;
        Xs[c * kLdS + r] = (r < nr && c < cols) ? B[(long long)c * ldb + r0 + r] : 0.f;
    }
    __syncthreads();
    for (int j = 0; j < nb; ++j) {
        const int cj = min(kT, cols - j * kT);
        float acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = Xs[(j * kT + tx * 4 + b) * kLdS + ty * 4 + a];
        for (int i = 0; i < j; ++i) {
            // Bs[k][c] = L_ji(c, k) = L(j*64 + c, i*64 + k)
            load_kmajor(Bs, L + (long long)(i * kT) * ldl + j * kT, ldl, cj, kT);
            __syncthreads();
            float p[4][4] = {};
            tile_mma(p, Xs + i * kT * kLdS, Bs);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] -= p[a][b];
            __syncthreads();
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) Ts[(tx * 4 + b) * kLdS + ty * 4 + a] = acc[a][b];
        load_kmajor(Bs, inv + (long long)j * kT * kT, kT, kT, kT);  // Bs[k][c] = D_j(c, k)
        __syncthreads();
        float x[4][4] = {};
        tile_mma(x, Ts, Bs);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
                Xs[(j * kT + tx * 4 + b) * kLdS + ty * 4 + a] = (tx * 4 + b < cj) ? x[a][b] : 0.f;
        __syncthreads();
    }
    for (int q = tid; q < kMaxRows * kT; q += kThreads) {
        const int c = q >> 6, r = q & 63;
        if (r < nr && c < cols) B[(long long)c * ldb + r0 + r] = Xs[c * kLdS + r];
    }
}

constexpr size_t kSmem = sizeof(float) * ((size_t)kMaxRows * kLdS + 2 * (size_t)kT * kLdS);
// llu_block_kernel<CW>: Xs (kMaxRows x (16 CW + 4)), As (64 x kLdS), Ts (64 x (16 CW + 4))
template <int CW>
constexpr size_t llu_smem()
{
    return sizeof(float) * ((size_t)kMaxRows * (16 * CW + 4) + (size_t)kT * kLdS +
                            (size_t)kT * (16 * CW + 4));
}

}  // namespace

int llu_block_max_rows() { return kMaxRows; }

void configure_trsm_block_kernels(hdbf_context*)
{
    cudaFuncSetAttribute(llu_block_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)llu_smem<4>());
    cudaFuncSetAttribute(llu_block_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)llu_smem<1>());
    cudaFuncSetAttribute(rlt_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    cudaGetLastError();
}

// B(rows x cols) <- B L^{-T} for non-unit lower L (cols <= 256); inv holds the
// 64x64 diagonal-block inverses of L (tri_inv64 layout).
hdbf_status rlt_block(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                      const float* inv, float* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    if (cols > kMaxRows) return HDBF_STATUS_INVALID_VALUE;
    const long long grid = ((long long)rows + kT - 1) / kT;
    ProfScope prof(ctx, kClsTrsmR, (double)cols * cols * rows, 8.0 * (double)rows * cols, rows,
                   cols, (cols + kT - 1) / kT);
    rlt_block_kernel<<<(unsigned)grid, kThreads, kSmem, ctx->stream>>>(rows, cols, L, ldl, inv, B,
                                                                      ldb);
    ctx->launches++;
    return last_cuda(ctx);
}

// B(rows x cols) <- L^{-1} B for unit lower L (rows <= 256); inv holds the
// 64x64 unit-lower diagonal-block inverses of L (tri_inv64 layout).
hdbf_status llu_block(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                      const float* inv, float* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    if (rows > kMaxRows) return HDBF_STATUS_INVALID_VALUE;
    const int nb = (rows + kT - 1) / kT;
    ProfScope prof(ctx, kClsTrsmL, (double)rows * rows * cols, 8.0 * (double)rows * cols, rows,
                   cols, nb);
    // 64 columns per CTA when that fills the SMs, else 16 (four times the CTAs)
    if ((cols + kT - 1) / kT >= ctx->sm_count) {
        const long long grid = ((long long)cols + 63) / 64;
        llu_block_kernel<4><<<(unsigned)grid, kThreads, llu_smem<4>(), ctx->stream>>>(
            rows, cols, L, ldl, inv, B, ldb);
    } else {
        const long long grid = ((long long)cols + 15) / 16;
        llu_block_kernel<1><<<(unsigned)grid, kThreads, llu_smem<1>(), ctx->stream>>>(
            rows, cols, L, ldl, inv, B, ldb);
    }
    ctx->launches++;
    return last_cuda(ctx);
}

}  // namespace hdbf
