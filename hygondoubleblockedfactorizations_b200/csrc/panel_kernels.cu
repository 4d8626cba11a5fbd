// Diagonal-block Cholesky and small triangular-solve kernels (FP32).
//
// potf2_small replaces rocsolver_spotrf on the diagonal block
// (src/potrf/double_blocked_potrf.cpp:34-56, call :334) at the leaf of this
// library's recursive diagonal factorization; tri_inv64 + {llu,rlt}_apply
// replace rocblas_strsm at the leaves of the recursive TRSMs
// (src/trsm/right_lower_trsm.cpp:24-37, src/getrf/getrf_npvt_internal.h:57-70).
#include <cfloat>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int kLeaf = 64;

// Right-looking Cholesky of an n x n (n <= 64) lower block, register
// resident: thread (r, g) = (tid % 64, tid / 64) holds A(r, g + 4i), i < 16.
// Per column j the owner group publishes the scaled column to shared memory
// and every thread applies the rank-1 update to its own 16 entries (two
// barriers per column, no shared-memory read-modify-write chains).
// Pivot test and info follow LAPACK xPOTRF: the first column whose updated
// diagonal is not > 0 (or is NaN) stops the factorization, its value is left
// in place, and info = info_base + j + 1 (first failure wins).  A block whose
// info is already non-zero is left untouched.
__global__ void __launch_bounds__(256) potf2_kernel(int n, float* A, long long lda, int* info,
                                                    int info_base)
{
    __shared__ float lcol[kLeaf];
    __shared__ float s_d;
    const int tid = threadIdx.x;
    const int r = tid & 63;
    const int g = tid >> 6;
    if (info && *reinterpret_cast<volatile int*>(info) != 0) return;

    float a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int c = g + 4 * i;
        a[i] = (r < n && c < n && r >= c) ? A[(long long)c * lda + r] : 0.f;
    }

    int failed_at = -1;
    for (int j = 0; j < n; ++j) {
        const int gj = j & 3, ij = j >> 2;
        float own = 0.f;
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (i == ij) own = a[i];
        if (g == gj && r == j) s_d = own;
        __syncthreads();
        const float d = s_d;
        if (!(d > 0.f)) {  // uniform: every thread read the same value
            failed_at = j;
            break;
        }
        const float sd = sqrtf(d);
        const float rcp = 1.0f / sd;
        if (g == gj) {
            const float v = (r == j) ? sd : (r > j ? own * rcp : own);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (i == ij) a[i] = v;
            if (r > j) lcol[r] = v;
        }
        __syncthreads();
        if (r > j) {
            const float lr = lcol[r];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int c = g + 4 * i;
                if (c > j && c <= r) a[i] = fmaf(-lr, lcol[c], a[i]);
            }
        }
    }

#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int c = g + 4 * i;
        if (r < n && c < n && r >= c) A[(long long)c * lda + r] = a[i];
    }
    if (failed_at >= 0 && tid == 0 && info) atomicCAS(info, 0, info_base + failed_at + 1);
}


// Inverses of the 64x64 diagonal blocks of a lower-triangular n x n matrix
// (unit or non-unit diagonal), one CTA per block, thread t solving
// L_bb x = e_t by forward substitution (right-looking, so every L read is a
// shared-memory broadcast).  out[b*4096 + c*64 + r] = inv(L_bb)(r, c); a
// partial last block is padded with the identity.
// mode 0: lower non-unit, 1: lower unit, 2: upper non-unit (the upper block
// U is inverted as (U^T)^{-1} and stored transposed).
__global__ void __launch_bounds__(kLeaf) tri_inv64_kernel(int n, const float* __restrict__ L,
                                                          long long ldl, int mode, float* out)
{
    __shared__ float Ls[kLeaf][kLeaf + 1];  // Ls[r][c] = T(base + r, base + c), T lower
    const int base = blockIdx.x * kLeaf;
    const int nb = min(kLeaf, n - base);
    const int t = threadIdx.x;
    const int unit = mode == 1;
    for (int idx = t; idx < kLeaf * kLeaf; idx += kLeaf) {
        const int c = idx / kLeaf, r = idx - c * kLeaf;
        float v = 0.f;
        if (r < nb && c < nb && r >= c)
            v = mode == 2 ? L[(long long)(base + r) * ldl + base + c]
                          : L[(long long)(base + c) * ldl + base + r];
        Ls[r][c] = v;
    }
    __syncthreads();
    float x[kLeaf];
#pragma unroll
    for (int i = 0; i < kLeaf; ++i) x[i] = (i == t) ? 1.f : 0.f;
#pragma unroll
    for (int k = 0; k < kLeaf; ++k) {
        if (k < nb) {
            if (!unit) x[k] = x[k] / Ls[k][k];
#pragma unroll
            for (int i = k + 1; i < kLeaf; ++i) x[i] = fmaf(-Ls[i][k], x[k], x[i]);
        }
    }
    float* ob = out + (long long)blockIdx.x * kLeaf * kLeaf;
    if (mode == 2) {
#pragma unroll
        for (int i = 0; i < kLeaf; ++i) ob[(long long)i * kLeaf + t] = x[i];  // row t of U^{-1}
    } else {
#pragma unroll
        for (int i = 0; i < kLeaf; ++i) ob[(long long)t * kLeaf + i] = x[i];  // column t
    }
}

// B(rows x cols) <- inv * B for rows <= 64 (inv = L^{-1} of the leaf block):
// CTA = 64 x 64 tile of B, thread = 4 x 4 outputs, in place.
__global__ void __launch_bounds__(256) llu_apply_kernel(int rows, int cols,
                                                        const float* __restrict__ inv, float* B,
                                                        long long ldb, int trans)
{
    __shared__ __align__(16) float Is[kLeaf][kLeaf];  // Is[k][r] = inv(r, k)
    __shared__ __align__(16) float Bs[kLeaf][kLeaf];  // Bs[k][c] = B(k, c0 + c)
    const int tid = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * kLeaf;
    for (int idx = tid; idx < kLeaf * kLeaf; idx += 256) {
        const int k = idx >> 6, r = idx & 63;
        Is[k][r] = trans ? inv[r * kLeaf + k] : inv[idx];
        const int c = idx >> 6, kk = idx & 63;
        Bs[kk][c] = (kk < rows && c0 + c < cols) ? B[(c0 + c) * ldb + kk] : 0.f;
    }
    __syncthreads();
    const int ty = tid >> 4, tx = tid & 15;
    float acc[4][4] = {};
#pragma unroll 16
    for (int k = 0; k < kLeaf; ++k) {
        const float4 a = *reinterpret_cast<const float4*>(&Is[k][ty * 4]);
        const float4 b = *reinterpret_cast<const float4*>(&Bs[k][tx * 4]);
        const float av[4] = {a.x, a.y, a.z, a.w};
        const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const long long c = c0 + tx * 4 + j;
        if (c >= cols) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = ty * 4 + i;
            if (r < rows) B[c * ldb + r] = acc[i][j];
        }
    }
}

// B(rows x cols) <- B * inv^T for cols <= 64 (inv = L^{-1} of the leaf
// block): CTA = 128 x 64 tile of B, thread = 8 rows x 4 columns, in place.
__global__ void __launch_bounds__(256) rlt_apply_kernel(int rows, int cols,
                                                        const float* __restrict__ inv, float* B,
                                                        long long ldb)
{
    __shared__ __align__(16) float Bs[kLeaf][128];   // Bs[k][r] = B(r0 + r, k)
    __shared__ __align__(16) float Is[kLeaf][kLeaf];  // Is[k][c] = inv(c, k)
    const int tid = threadIdx.x;
    const long long r0 = (long long)blockIdx.x * 128;
    for (int idx = tid; idx < kLeaf * kLeaf; idx += 256) Is[idx >> 6][idx & 63] = inv[idx];
    for (int idx = tid; idx < kLeaf * 128; idx += 256) {
        const int k = idx >> 7, r = idx & 127;
        Bs[k][r] = (k < cols && r0 + r < rows) ? B[(long long)k * ldb + r0 + r] : 0.f;
    }
    __syncthreads();
    const int ty = tid >> 4, tx = tid & 15;
    float acc[8][4] = {};
#pragma unroll 8
    for (int k = 0; k < kLeaf; ++k) {
        const float4 a0 = *reinterpret_cast<const float4*>(&Bs[k][ty * 8]);
        const float4 a1 = *reinterpret_cast<const float4*>(&Bs[k][ty * 8 + 4]);
        const float4 b = *reinterpret_cast<const float4*>(&Is[k][tx * 4]);
        const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int c = tx * 4 + j;
        if (c >= cols) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const long long r = r0 + ty * 8 + i;
            if (r < rows) B[(long long)c * ldb + r] = acc[i][j];
        }
    }
}

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

hdbf_status tri_inv64(hdbf_context* ctx, int n, const float* L, long long ldl, bool unit,
                      float* out)
{
    return tri_inv64_mode(ctx, n, L, ldl, unit ? 1 : 0, out);
}

hdbf_status tri_inv64_mode(hdbf_context* ctx, int n, const float* L, long long ldl, int mode,
                           float* out)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    const int blocks = (n + kLeaf - 1) / kLeaf;
    ProfScope prof(ctx, kClsTrsmInv, (double)blocks * kLeaf * kLeaf * kLeaf / 3.0,
                   8.0 * blocks * kLeaf * kLeaf);
    tri_inv64_kernel<<<blocks, kLeaf, 0, ctx->stream>>>(n, L, ldl, mode, out);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status llu_apply(hdbf_context* ctx, int rows, int cols, const float* inv, float* B,
                      long long ldb)
{
    return llu_apply_t(ctx, rows, cols, inv, B, ldb, false);
}

hdbf_status llu_apply_t(hdbf_context* ctx, int rows, int cols, const float* inv, float* B,
                        long long ldb, bool trans)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    if (rows > kLeaf) return HDBF_STATUS_INVALID_VALUE;
    const long long grid = ((long long)cols + kLeaf - 1) / kLeaf;
    ProfScope prof(ctx, kClsTrsmL, 2.0 * kLeaf * kLeaf * (double)cols, 8.0 * rows * cols);
    llu_apply_kernel<<<(unsigned)grid, 256, 0, ctx->stream>>>(rows, cols, inv, B, ldb,
                                                               trans ? 1 : 0);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status rlt_apply(hdbf_context* ctx, int rows, int cols, const float* inv, float* B,
                      long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    if (cols > kLeaf) return HDBF_STATUS_INVALID_VALUE;
    const long long grid = ((long long)rows + 127) / 128;
    ProfScope prof(ctx, kClsTrsmR, 2.0 * kLeaf * kLeaf * (double)rows, 8.0 * rows * cols);
    rlt_apply_kernel<<<(unsigned)grid, 256, 0, ctx->stream>>>(rows, cols, inv, B, ldb);
    ctx->launches++;
    return last_cuda(ctx);
}

}  // namespace hdbf
