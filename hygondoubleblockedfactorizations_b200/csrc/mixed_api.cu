// C ABI: mixed-precision GEMM entry point (tensor cores).
#include <algorithm>

#include "internal.h"
#include "gemm/mixed_gemm.h"

namespace hdbf {
namespace {

__global__ void scale_cols_kernel(float* C, int m, int n, long long ldc, float beta)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const long long c = blockIdx.y;
    if (r < m && c < n) C[c * ldc + r] = beta == 0.f ? 0.f : beta * C[c * ldc + r];
}

inline long long pad8(long long x) { return (x + 7) / 8 * 8; }

// C = alpha * op(A) * op(B) + beta * C with FP16 operands rounded once into
// K-major shadows (reference semantics: src/gemm/mixed_gemm.cpp:8-96, FP16
// inputs; here C stays FP32 and accumulation is FP32 in TMEM).
hdbf_status mixed_gemm_impl(hdbf_context* ctx, bool ta, bool tb, int m, int n, int k, float alpha,
                            const float* A, long long lda, const float* B, long long ldb,
                            float beta, float* C, long long ldc)
{
    if (m < 0 || n < 0 || k < 0) return HDBF_STATUS_INVALID_VALUE;
    if (m == 0 || n == 0) return HDBF_STATUS_SUCCESS;
    if (!C || ldc < std::max(1, m)) return HDBF_STATUS_INVALID_VALUE;
    if (beta != 1.f) {
        dim3 grid((m + 255) / 256, n);
        scale_cols_kernel<<<grid, 256, 0, ctx->stream>>>(C, m, n, ldc, beta);
        ctx->launches++;
        HDBF_TRY(last_cuda(ctx));
    }
    if (k == 0 || alpha == 0.f) return HDBF_STATUS_SUCCESS;
    if (!A || !B) return HDBF_STATUS_INVALID_VALUE;
    const long long kp = pad8(k);
    hdbf_status st;
    char* arena = static_cast<char*>(mixed_arena(ctx, (size_t)(m + n) * kp * 2 + 256, &st));
    if (!arena) return st;
    void* sa = arena;
    void* sb = arena + (size_t)m * kp * 2;
    // op(A) is m x k; K-major shadow row i = row i of op(A).
    if (!ta) HDBF_TRY(convert_transpose16(ctx, kFmtF16, m, k, A, lda, sa, nullptr, kp, 1.f));
    else HDBF_TRY(convert_direct16(ctx, kFmtF16, k, m, A, lda, sa, nullptr, kp, 1.f));
    // op(B) is k x n; shadow row j = column j of op(B).
    if (!tb) HDBF_TRY(convert_direct16(ctx, kFmtF16, k, n, B, ldb, sb, nullptr, kp, 1.f));
    else HDBF_TRY(convert_transpose16(ctx, kFmtF16, n, k, B, ldb, sb, nullptr, kp, 1.f));
    TcOperand oa, ob;
    oa.base = sa;
    oa.ld = kp;
    ob.base = sb;
    ob.ld = kp;
    return tc_gemm_sub(ctx, kFmtF16, m, n, k, oa, ob, C, ldc, -alpha, false);
}

}  // namespace
}  // namespace hdbf

using namespace hdbf;

extern "C" {

void launch_mixed_gemm(hdbf_handle handle, cudaStream_t stream, rocblas_operation transA,
                       rocblas_operation transB, int m, int n, int k, float alpha,
                       const float* A_f32, int lda, const float* B_f32, int ldb, float beta,
                       float* C_f32, int ldc)
{
    if (!handle) return;
    cudaStream_t saved = handle->stream;
    handle->stream = stream;
    handle->last_status =
        mixed_gemm_impl(handle, transA != rocblas_operation_none, transB != rocblas_operation_none,
                        m, n, k, alpha, A_f32, lda, B_f32, ldb, beta, C_f32, ldc);
    handle->stream = saved;
}

}  // extern "C"
