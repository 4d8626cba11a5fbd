// Diagonal-block Cholesky and small triangular-solve kernels (FP32).
//
// potf2_small replaces rocsolver_spotrf on the diagonal block
// (src/potrf/double_blocked_potrf.cpp:34-56, call :334) at the leaf of this
// library's recursive diagonal factorization; trsm_*_small replace
// rocblas_strsm at the leaves of the recursive TRSMs
// (src/trsm/right_lower_trsm.cpp:24-37, src/getrf/getrf_npvt_internal.h:57-70).
#include <cfloat>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int kLeaf = 64;

// Right-looking Cholesky of an n x n (n <= 64) lower block held in shared
// memory.  Pivot test and info follow LAPACK xPOTRF: the first column whose
// updated diagonal is not > 0 (or is NaN) stops the factorization, its value
// is left in place, and info = info_base + j + 1 (first failure wins).  A
// block whose info is already non-zero is left untouched.
__global__ void __launch_bounds__(256) potf2_kernel(int n, float* A, long long lda, int* info,
                                                    int info_base)
{
    __shared__ float s[kLeaf][kLeaf + 1];  // s[col][row]
    __shared__ float s_diag;
    const int tid = threadIdx.x;
    if (info && *reinterpret_cast<volatile int*>(info) != 0) return;

    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int c = idx / n, r = idx - c * n;
        if (r >= c) s[c][r] = A[(long long)c * lda + r];
    }
    __syncthreads();

    int failed_at = -1;
    for (int j = 0; j < n; ++j) {
        const float d = s[j][j];
        __syncthreads();
        if (!(d > 0.f)) {  // uniform: every thread read the same value
            failed_at = j;
            break;
        }
        const float sd = sqrtf(d);
        const float rcp = 1.0f / sd;
        if (tid == 0) s[j][j] = sd;
        for (int i = j + 1 + tid; i < n; i += blockDim.x) s[j][i] *= rcp;
        __syncthreads();
        // trailing lower update: s[c][r] -= s[j][r] * s[j][c], j < c <= r
        const int tc = tid >> 6, tr = tid & 63;
        for (int c = j + 1 + tc; c < n; c += 4) {
            const float ljc = s[j][c];
            for (int r = c + tr; r < n; r += 64) s[c][r] -= s[j][r] * ljc;
        }
        __syncthreads();
    }

    for (int idx = tid; idx < n * n; idx += blockDim.x) {
        const int c = idx / n, r = idx - c * n;
        if (r >= c) A[(long long)c * lda + r] = s[c][r];
    }
    if (failed_at >= 0 && tid == 0 && info) atomicCAS(info, 0, info_base + failed_at + 1);
}

// B(rows x cols) <- B * L^{-T} (cols <= 64): one thread per row, the row held
// in registers, L broadcast from shared memory.  Column order and the
// reciprocal-of-diagonal scaling follow reference BLAS xTRSM (Right, Lower,
// Transposed, Non-unit).
constexpr int kRltThreads = 128;
__global__ void __launch_bounds__(kRltThreads) trsm_rlt_kernel(int rows, int cols,
                                                               const float* __restrict__ L,
                                                               long long ldl, float* B,
                                                               long long ldb)
{
    __shared__ float Ls[kLeaf][kLeaf];  // Ls[c][r] = L(r, c)
    __shared__ float rd[kLeaf];
    const int tid = threadIdx.x;
    for (int idx = tid; idx < kLeaf * kLeaf; idx += blockDim.x) {
        const int c = idx / kLeaf, r = idx - c * kLeaf;
        Ls[c][r] = (r < cols && c < cols && r >= c) ? L[(long long)c * ldl + r] : 0.f;
    }
    __syncthreads();
    for (int c = tid; c < kLeaf; c += blockDim.x) rd[c] = (c < cols) ? 1.0f / Ls[c][c] : 0.f;
    __syncthreads();

    const long long row = (long long)blockIdx.x * kRltThreads + tid;
    if (row >= rows) return;
    float x[kLeaf];
#pragma unroll
    for (int j = 0; j < kLeaf; ++j) x[j] = (j < cols) ? B[(long long)j * ldb + row] : 0.f;
#pragma unroll
    for (int k = 0; k < kLeaf; ++k) {
        if (k < cols) {
            x[k] *= rd[k];
#pragma unroll
            for (int j = k + 1; j < kLeaf; ++j) x[j] = fmaf(-Ls[k][j], x[k], x[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < kLeaf; ++j)
        if (j < cols) B[(long long)j * ldb + row] = x[j];
}

// B(rows x cols) <- L^{-1} B, L unit lower (rows <= 64): one thread per
// column; the CTA's 128 columns are staged through shared memory so global
// traffic stays coalesced down each column.
constexpr int kLluCols = 128;
__global__ void __launch_bounds__(kLluCols) trsm_llu_kernel(int rows, int cols,
                                                            const float* __restrict__ L,
                                                            long long ldl, float* B,
                                                            long long ldb)
{
    extern __shared__ float sm[];
    float* Ls = sm;                       // [kLeaf][kLeaf]  Ls[c*64 + r] = L(r, c)
    float* Bs = sm + kLeaf * kLeaf;       // [kLeaf][kLluCols + 1]
    constexpr int BST = kLluCols + 1;
    const int tid = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * kLluCols;
    for (int idx = tid; idx < kLeaf * kLeaf; idx += blockDim.x) {
        const int c = idx / kLeaf, r = idx - c * kLeaf;
        Ls[idx] = (r < rows && c < rows && r > c) ? L[(long long)c * ldl + r] : 0.f;
    }
    for (int idx = tid; idx < rows * kLluCols; idx += blockDim.x) {
        const int c = idx / rows, r = idx - c * rows;
        const long long gc = c0 + c;
        Bs[r * BST + c] = (gc < cols) ? B[gc * ldb + r] : 0.f;
    }
    __syncthreads();
    float x[kLeaf];
#pragma unroll
    for (int r = 0; r < kLeaf; ++r) x[r] = (r < rows) ? Bs[r * BST + tid] : 0.f;
#pragma unroll
    for (int p = 0; p < kLeaf; ++p) {
        if (p < rows) {
#pragma unroll
            for (int i = p + 1; i < kLeaf; ++i) x[i] = fmaf(-Ls[p * kLeaf + i], x[p], x[i]);
        }
    }
#pragma unroll
    for (int r = 0; r < kLeaf; ++r)
        if (r < rows) Bs[r * BST + tid] = x[r];
    __syncthreads();
    for (int idx = tid; idx < rows * kLluCols; idx += blockDim.x) {
        const int c = idx / rows, r = idx - c * rows;
        const long long gc = c0 + c;
        if (gc < cols) B[gc * ldb + r] = Bs[r * BST + c];
    }
}

constexpr size_t kLluSmem = (size_t)(kLeaf * kLeaf + kLeaf * (kLluCols + 1)) * sizeof(float);

}  // namespace

hdbf_status potf2_small(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                        int info_base)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    if (n > kLeaf) return HDBF_STATUS_INVALID_VALUE;
    ProfScope prof(ctx, kClsPotf2, (double)n * n * n / 3.0, 8.0 * n * n);
    potf2_kernel<<<1, 256, 0, ctx->stream>>>(n, A, lda, info, info_base);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status trsm_rlt_small(hdbf_context* ctx, int rows, int cols, const float* L,
                           long long ldl, float* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    if (cols > kLeaf) return HDBF_STATUS_INVALID_VALUE;
    const long long grid = ((long long)rows + kRltThreads - 1) / kRltThreads;
    ProfScope prof(ctx, kClsTrsmR, (double)rows * cols * cols, 8.0 * rows * cols);
    trsm_rlt_kernel<<<(unsigned)grid, kRltThreads, 0, ctx->stream>>>(rows, cols, L, ldl, B,
                                                                      ldb);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status trsm_llu_small(hdbf_context* ctx, int rows, int cols, const float* L,
                           long long ldl, float* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    if (rows > kLeaf) return HDBF_STATUS_INVALID_VALUE;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(trsm_llu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kLluSmem);
        configured = true;
    }
    const long long grid = ((long long)cols + kLluCols - 1) / kLluCols;
    ProfScope prof(ctx, kClsTrsmL, (double)cols * rows * rows, 8.0 * rows * cols);
    trsm_llu_kernel<<<(unsigned)grid, kLluCols, kLluSmem, ctx->stream>>>(rows, cols, L, ldl,
                                                                         B, ldb);
    ctx->launches++;
    return last_cuda(ctx);
}

}  // namespace hdbf
