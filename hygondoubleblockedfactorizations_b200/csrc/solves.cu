// Triangular solves with several right-hand sides (POTRS / GETRS) on the
// FP32 factors.  Not part of the reference (it has no solve); needed by the
// iterative-refinement driver.  The 64x64 diagonal blocks of the triangle are
// inverted once per solve.  Up to kWaveMaxRhs right-hand sides, each
// triangle is one wavefront launch (trsm_wave.cu); wider right-hand sides use
// the recursion on row halves with GEMM updates and inverse leaves.
#include <algorithm>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int kLeaf = 64;
constexpr int kWaveMaxRhs = 64;

inline int split_at(int n)
{
    int h = (n / 2 + kLeaf - 1) / kLeaf * kLeaf;
    if (h <= 0 || h >= n) h = n > kLeaf ? n - kLeaf : 1;
    return h;
}

inline const float* blk(const float* inv, int row0) { return inv + (long long)(row0 / kLeaf) * 4096; }

// L X = B, L lower (unit or not): forward.
hdbf_status fwd_lower(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                      float* B, long long ldb, const float* inv)
{
    if (rows <= kLeaf) return llu_apply_t(ctx, rows, cols, inv, B, ldb, false);
    const int r1 = split_at(rows), r2 = rows - r1;
    HDBF_TRY(fwd_lower(ctx, r1, cols, L, ldl, B, ldb, inv));
    HDBF_TRY(sgemm_sub(ctx, true, false, r2, cols, r1, L + r1, ldl, B, ldb, B + r1, ldb));
    return fwd_lower(ctx, r2, cols, L + (long long)r1 * ldl + r1, ldl, B + r1, ldb, blk(inv, r1));
}

// U X = B, U upper non-unit: backward.
hdbf_status bwd_upper(hdbf_context* ctx, int rows, int cols, const float* U, long long ldu,
                      float* B, long long ldb, const float* inv)
{
    if (rows <= kLeaf) return llu_apply_t(ctx, rows, cols, inv, B, ldb, false);
    const int r1 = split_at(rows), r2 = rows - r1;
    HDBF_TRY(bwd_upper(ctx, r2, cols, U + (long long)r1 * ldu + r1, ldu, B + r1, ldb,
                       blk(inv, r1)));
    HDBF_TRY(sgemm_sub(ctx, true, false, r1, cols, r2, U + (long long)r1 * ldu, ldu, B + r1, ldb,
                       B, ldb));
    return bwd_upper(ctx, r1, cols, U, ldu, B, ldb, inv);
}

// L^T X = B, L lower non-unit: backward with the transposed triangle.
hdbf_status bwd_lower_t(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                        float* B, long long ldb, const float* inv)
{
    if (rows <= kLeaf) return llu_apply_t(ctx, rows, cols, inv, B, ldb, true);
    const int r1 = split_at(rows), r2 = rows - r1;
    HDBF_TRY(bwd_lower_t(ctx, r2, cols, L + (long long)r1 * ldl + r1, ldl, B + r1, ldb,
                         blk(inv, r1)));
    // B1 -= L21^T X2, L21 = L(r1:rows, 0:r1) is r2 x r1
    HDBF_TRY(sgemm_sub_tn(ctx, r1, cols, r2, L + r1, ldl, B + r1, ldb, B, ldb));
    return bwd_lower_t(ctx, r1, cols, L, ldl, B, ldb, inv);
}

// Full row permutation from LAPACK pivots: perm[i] = original row now at row i.
__global__ void __launch_bounds__(1024) ipiv_to_perm_kernel(const int* ipiv, int n, int* perm,
                                                            int use_smem)
{
    extern __shared__ int sp[];
    int* p = use_smem ? sp : perm;
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = i;
    __syncthreads();
    // The swaps are a dependent chain; warp 0 loads the next 32 pivots
    // while lane 0 applies the current 32 (pivots arrive by shuffle).
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int cur = lane < n ? ipiv[lane] : 0;
        for (int i0 = 0; i0 < n; i0 += 32) {
            const int nx = i0 + 32 + lane < n ? ipiv[i0 + 32 + lane] : 0;
            const int cnt = n - i0 < 32 ? n - i0 : 32;
            for (int u = 0; u < cnt; ++u) {
                const int b = __shfl_sync(0xffffffffu, cur, u) - 1;
                const int i = i0 + u;
                if (lane == 0 && b != i && b >= 0 && b < n) {
                    const int t = p[i];
                    p[i] = p[b];
                    p[b] = t;
                }
                __syncwarp();
            }
            cur = nx;
        }
    }
    __syncthreads();
    if (use_smem)
        for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = p[i];
}

__global__ void gather_rows_perm_kernel(const float* __restrict__ src, long long lds, float* dst,
                                        long long ldd, const int* __restrict__ perm, int n,
                                        int cols)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const long long c = blockIdx.y;
    if (r < n && c < cols) dst[c * ldd + r] = src[c * lds + perm[r]];
}

}  // namespace

hdbf_status ipiv_to_perm(hdbf_context* ctx, const int* ipiv, int n, int* perm)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    const size_t smem = (size_t)n * sizeof(int);
    const size_t cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    const int use = smem <= cap ? 1 : 0;
    ProfScope prof(ctx, kClsCompose, 0.0, 12.0 * n);
    ipiv_to_perm_kernel<<<1, 1024, use ? smem : 0, ctx->stream>>>(ipiv, n, perm, use);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status gather_rows_perm(hdbf_context* ctx, const float* src, long long lds, float* dst,
                             long long ldd, const int* perm, int n, int cols)
{
    if (n <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    dim3 grid((n + 255) / 256, cols);
    ProfScope prof(ctx, kClsMoves, 0.0, 8.0 * n * cols);
    gather_rows_perm_kernel<<<grid, 256, 0, ctx->stream>>>(src, lds, dst, ldd, perm, n, cols);
    ctx->launches++;
    return last_cuda(ctx);
}

void configure_solve_kernels(hdbf_context* ctx)
{
    const size_t cap = ctx->max_smem_optin > 4096 ? ctx->max_smem_optin - 4096 : 0;
    cudaFuncSetAttribute(ipiv_to_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap);
    cudaGetLastError();
    configure_wave_kernels(ctx);
}

// B <- L^{-T} L^{-1} B for the Cholesky factor L (lower, non-unit).
hdbf_status potrs_f32(hdbf_context* ctx, const float* L, long long ldl, int n, int nrhs, float* B,
                      long long ldb)
{
    if (n <= 0 || nrhs <= 0) return HDBF_STATUS_SUCCESS;
    HDBF_TRY(ensure_ws(ctx, n));
    float* inv = ws_inv(ctx);
    HDBF_TRY(tri_inv64_mode(ctx, n, L, ldl, 0, inv));
    if (nrhs <= kWaveMaxRhs) {
        HDBF_TRY(trsv_wave(ctx, n, nrhs, L, ldl, false, inv, false, B, ldb));
        return trsv_wave(ctx, n, nrhs, L, ldl, true, inv, true, B, ldb);
    }
    HDBF_TRY(fwd_lower(ctx, n, nrhs, L, ldl, B, ldb, inv));
    return bwd_lower_t(ctx, n, nrhs, L, ldl, B, ldb, inv);
}

// B <- U^{-1} L^{-1} B' where B' = P B was formed by the caller (the
// permutation is applied out of place with gather_rows_perm).
hdbf_status getrs_f32_permuted(hdbf_context* ctx, const float* LU, long long ldlu, int n, int nrhs,
                               float* B, long long ldb)
{
    if (n <= 0 || nrhs <= 0) return HDBF_STATUS_SUCCESS;
    HDBF_TRY(ensure_ws(ctx, n));
    float* inv = ws_inv(ctx);
    const bool wave = nrhs <= kWaveMaxRhs;
    HDBF_TRY(tri_inv64_mode(ctx, n, LU, ldlu, 1, inv));
    if (wave) HDBF_TRY(trsv_wave(ctx, n, nrhs, LU, ldlu, false, inv, false, B, ldb));
    else HDBF_TRY(fwd_lower(ctx, n, nrhs, LU, ldlu, B, ldb, inv));
    HDBF_TRY(tri_inv64_mode(ctx, n, LU, ldlu, 2, inv));
    if (wave) return trsv_wave(ctx, n, nrhs, LU, ldlu, false, inv, true, B, ldb);
    return bwd_upper(ctx, n, nrhs, LU, ldlu, B, ldb, inv);
}

}  // namespace hdbf
