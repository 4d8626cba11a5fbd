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

__global__ void __launch_bounds__(kThreads) llu_block_kernel(int rows, int cols,
                                                             const float* __restrict__ L,
                                                             long long ldl,
                                                             const float* __restrict__ inv,
                                                             float* B, long long ldb)
{
    extern __shared__ __align__(16) float sm[];
    float* Xs = sm;                       // kMaxRows x kLdS: Xs[r][c] = B(r, c0 + c)
    float* As = Xs + kMaxRows * kLdS;     // left operand tile
    float* Ts = As + kT * kLdS;           // right operand staging
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const long long c0 = (long long)blockIdx.x * kT;
    const int nc = (int)min((long long)kT, (long long)cols - c0);
    const int nb = (rows + kT - 1) / kT;

    for (int q = tid; q < kMaxRows * kT; q += kThreads) {
        const int c = q / kMaxRows, r = q - c * kMaxRows;
        Xs[r * kLdS + c] = (r < rows && c < nc) ? B[(c0 + c) * ldb + r] : 0.f;
    }
    __syncthreads();
    for (int i = 0; i < nb; ++i) {
        const int ri = min(kT, rows - i * kT);
        float acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = Xs[(i * kT + ty * 4 + a) * kLdS + tx * 4 + b];
        for (int j = 0; j < i; ++j) {
            load_kmajor(As, L + (long long)(j * kT) * ldl + i * kT, ldl, ri, kT);
            __syncthreads();
            float p[4][4] = {};
            tile_mma(p, As, Xs + j * kT * kLdS);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] -= p[a][b];
            __syncthreads();
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) Ts[(ty * 4 + a) * kLdS + tx * 4 + b] = acc[a][b];
        load_kmajor(As, inv + (long long)i * kT * kT, kT, kT, kT);
        __syncthreads();
        float x[4][4] = {};
        tile_mma(x, As, Ts);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b)
                Xs[(i * kT + ty * 4 + a) * kLdS + tx * 4 + b] = (ty * 4 + a < ri) ? x[a][b] : 0.f;
        __syncthreads();
    }
    for (int q = tid; q < kMaxRows * kT; q += kThreads) {
        const int c = q / kMaxRows, r = q - c * kMaxRows;
        if (r < rows && c < nc) B[(c0 + c) * ldb + r] = Xs[r * kLdS + c];
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

}  // namespace

int llu_block_max_rows() { return kMaxRows; }

void configure_trsm_block_kernels(hdbf_context*)
{
    cudaFuncSetAttribute(llu_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
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
    const long long grid = ((long long)cols + kT - 1) / kT;
    const int nb = (rows + kT - 1) / kT;
    ProfScope prof(ctx, kClsTrsmL, (double)rows * rows * cols, 8.0 * (double)rows * cols, rows,
                   cols, nb);
    llu_block_kernel<<<(unsigned)grid, kThreads, kSmem, ctx->stream>>>(rows, cols, L, ldl, inv, B,
                                                                      ldb);
    ctx->launches++;
    return last_cuda(ctx);
}

}  // namespace hdbf
