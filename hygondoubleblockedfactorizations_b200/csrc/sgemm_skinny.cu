// Skinny FP32 update C (M x N, N <= 32) -= op(A) * op(B).
//
// The triangular solves with a few right-hand sides and the narrowest panel
// updates multiply a tall matrix by a thin one: the 128 x 128 register tile of
// sgemm_sub_kernel would waste up to 7/8 of its FMAs there, and the work is
// bound by reading A once.  Here each thread owns one row of C (all N
// columns in registers), streams its row of op(A) through a K loop, and reads
// the current K-chunk of op(B) from shared memory as broadcasts.  Long K is
// split across CTAs (grid.y) with FP32 partial sums reduced by a second
// kernel in a fixed order, so results do not depend on scheduling.
#include "internal.h"

namespace hdbf {
namespace {

constexpr int kRows = 256;  // rows of C per CTA (one per thread)
constexpr int kNB = 32;     // max columns
constexpr int kKC = 32;     // K chunk staged in shared memory

// mode: 0 NT (A M x K, B N x K), 1 NN (B K x N), 2 TN (A K x M, B K x N).
// NB is the column count rounded up to 8, 16 or 32.
template <int MODE, int NB>
__global__ void __launch_bounds__(kRows) skinny_kernel(int M, int N, int K, const float* __restrict__ A,
                                                       long long lda, const float* __restrict__ B,
                                                       long long ldb, float* C, long long ldc,
                                                       float* partial, int kper)
{
    __shared__ __align__(16) float Bs[kKC][NB];
    const int row = blockIdx.x * kRows + threadIdx.x;
    const int s = blockIdx.y;
    const int k0 = s * kper, k1 = min(K, k0 + kper);
    float acc[NB];
#pragma unroll
    for (int n = 0; n < NB; ++n) acc[n] = 0.f;
    for (int kb = k0; kb < k1; kb += kKC) {
        const int kn = min(kKC, k1 - kb);
        __syncthreads();
        for (int idx = threadIdx.x; idx < kKC * NB; idx += kRows) {
            int kc, n;
            if (MODE == 0) { kc = idx / NB; n = idx % NB; }
            else { n = idx / kKC; kc = idx % kKC; }
            float v = 0.f;
            if (kc < kn && n < N)
                v = MODE == 0 ? B[(long long)(kb + kc) * ldb + n] : B[(long long)n * ldb + kb + kc];
            Bs[kc][n] = v;
        }
        __syncthreads();
        if (row < M) {
            if (kn == kKC) {
#pragma unroll 8
                for (int kc = 0; kc < kKC; ++kc) {
                    const float a = MODE == 2 ? __ldg(A + (long long)row * lda + kb + kc)
                                              : __ldg(A + (long long)(kb + kc) * lda + row);
#pragma unroll
                    for (int n = 0; n < NB; ++n) acc[n] = fmaf(a, Bs[kc][n], acc[n]);
                }
            } else {
                for (int kc = 0; kc < kn; ++kc) {
                    const float a = MODE == 2 ? __ldg(A + (long long)row * lda + kb + kc)
                                              : __ldg(A + (long long)(kb + kc) * lda + row);
#pragma unroll
                    for (int n = 0; n < NB; ++n) acc[n] = fmaf(a, Bs[kc][n], acc[n]);
                }
            }
        }
    }
    if (row >= M) return;
    if (partial) {
#pragma unroll
        for (int n = 0; n < NB; ++n)
            if (n < N) partial[((long long)s * N + n) * M + row] = acc[n];
        return;
    }
    float cv[NB];
#pragma unroll
    for (int n = 0; n < NB; ++n) cv[n] = n < N ? C[(long long)n * ldc + row] : 0.f;
#pragma unroll
    for (int n = 0; n < NB; ++n)
        if (n < N) C[(long long)n * ldc + row] = cv[n] - acc[n];
}

__global__ void skinny_reduce_kernel(const float* __restrict__ partial, int S, int M, int N,
                                     float* C, long long ldc)
{
    const int row = blockIdx.x * 256 + threadIdx.x;
    const int n = blockIdx.y;
    if (row >= M || n >= N) return;
    float acc = 0.f;
    for (int s = 0; s < S; ++s) acc += partial[((long long)s * N + n) * M + row];
    C[(long long)n * ldc + row] -= acc;
}

}  // namespace

size_t skinny_partial_floats(int n) { return (size_t)8 * kNB * (size_t)(n < 1 ? 1 : n); }

hdbf_status sgemm_skinny(hdbf_context* ctx, int mode, int M, int N, int K, const float* A,
                         long long lda, const float* B, long long ldb, float* C, long long ldc)
{
    if (M <= 0 || N <= 0 || K <= 0) return HDBF_STATUS_SUCCESS;
    if (N > kNB) return HDBF_STATUS_INVALID_VALUE;
    const int gx = (M + kRows - 1) / kRows;
    int S = 1;
    while (S < 8 && gx * S < 2 * ctx->sm_count && K >= (S * 2) * 128) S *= 2;
    float* partial = nullptr;
    if (S > 1) {
        if (ctx->ws && ctx->ws_n >= M) partial = ws_skinny(ctx);
        else S = 1;
    }
    const int kper = (K + S - 1) / S;
    ProfScope prof(ctx, kClsSkinny, 2.0 * (double)M * N * K, 4.0 * ((double)M * K + 2.0 * M * N), M,
                   N, K);
    dim3 grid(gx, S);
    cudaStream_t st = ctx->stream;
#define HDBF_SKINNY(MD, NBV) \
    skinny_kernel<MD, NBV><<<grid, kRows, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, partial, kper)
#define HDBF_SKINNY_NB(MD)                    \
    if (N <= 8) HDBF_SKINNY(MD, 8);           \
    else if (N <= 16) HDBF_SKINNY(MD, 16);    \
    else HDBF_SKINNY(MD, 32)
    if (mode == 0) { HDBF_SKINNY_NB(0); }
    else if (mode == 1) { HDBF_SKINNY_NB(1); }
    else { HDBF_SKINNY_NB(2); }
#undef HDBF_SKINNY_NB
#undef HDBF_SKINNY
    ctx->launches++;
    if (S > 1) {
        dim3 g2((M + 255) / 256, N);
        skinny_reduce_kernel<<<g2, 256, 0, ctx->stream>>>(partial, S, M, N, C, ldc);
        ctx->launches++;
    }
    return last_cuda(ctx);
}

}  // namespace hdbf
