// FP64 building blocks behind the reference's `_double` entry points
// (include/potrf/double_blocked_potrf.h:57-103, include/getrf/
// double_blocked_getrf.h:37-74 and the SYRK / TRSM / GEMM twins).  The
// drivers in api_potrf.cu and api_getrf.cu are templates over the scalar
// type; this file gives them the FP64 overloads of their primitives:
//
//   gemm_sub / gemm_sub_tn   C -= op(A) op(B), FP64 FMA: 128x128x8 tiles with
//                            8x8 outputs per thread for large updates, 64x64x16
//                            with 4x4 for narrow ones; lower-triangle mode
//   potf2_small              <= 64 Cholesky leaf, one CTA, LAPACK info
//   tri_inv64                inverses of the 64x64 diagonal blocks
//   trsm_rlt / trsm_llu      recursive TRSMs with inverse-apply leaves
//   potrf_diag, syrk_lower   recursive diagonal Cholesky, lower SYRK
//   getrf_panel              recursive LU panel on the grid-wide leaf below
//   apply_moves              composed row moves, gathered through scratch
//
// The panel leaf (getf2_coop64_kernel, <= 64 columns) keeps ~256 rows per
// CTA in shared memory and runs one global exchange per column: every CTA
// writes its candidate (|a|, row, the candidate row and, from the owner, the
// diagonal row) into its slot and publishes a sequence number with a release
// store; every CTA polls all sequence numbers with acquire loads (bounded),
// picks the same winner (largest |a|, lowest row on ties -- LAPACK IDAMAX),
// swaps, scales by the reciprocal pivot (division when |pivot| < DBL_MIN, as
// xGETF2) and applies the rank-1 update to its own rows.  Sequence numbers
// are epoch * 256 + column + 1 (epoch = the panel launch counter shared with
// the FP32 leaf, column < 64), so no launch accepts another launch's slot.
#include <algorithm>
#include <cfloat>
#include <climits>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int kL = 64;  // leaf / diagonal-block order

inline int split64(int n)
{
    int h = (n / 2 + kL - 1) / kL * kL;
    if (h <= 0 || h >= n) h = std::max(1, n - kL);
    return h;
}

// ------------------------------------------------------------------ GEMM
// Large updates: 128x128x8 tiles, 256 threads, 8x8 outputs per thread in the split layout
// (rows ty*4 + {0..3} and 64 + ty*4 + {0..3}, columns likewise with tx), so
// every fragment is two 16-byte shared-memory loads; the next k-tile is
// copied into the other shared-memory buffer with 8-byte cp.async (zero fill
// outside the matrix) while the current one is consumed.
constexpr int GBM = 128, GBN = 128, GBK = 8, GTHR = 256, GLD = GBM + 4;

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem),
                 "r"(valid ? 8 : 0)
                 : "memory");
}

// MODE 0: C -= A B^T (A M x K, B N x K); 1: C -= A B (B K x N);
// 2: C -= A^T B (A stored K x M, B K x N).  TRI: only entries with row >= col
// (local to C) are written and tiles wholly above the diagonal are skipped.
template <int MODE, bool TRI>
__global__ void __launch_bounds__(GTHR, 1) dgemm_sub_kernel(int M, int N, int K,
                                                            const double* __restrict__ A,
                                                            long long lda,
                                                            const double* __restrict__ B,
                                                            long long ldb, double* C,
                                                            long long ldc, int tiles_m)
{
    __shared__ __align__(16) double As[2][GBK][GLD];  // As[buf][k][m]
    __shared__ __align__(16) double Bs[2][GBK][GLD];  // Bs[buf][k][n]
    const int tile = blockIdx.x;
    const int m0 = (tile % tiles_m) * GBM, n0 = (tile / tiles_m) * GBN;
    if (TRI && n0 >= m0 + GBM) return;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    double acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    auto issue = [&](int buf, int k0) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int q = tid + e * GTHR;
            int m, k;
            if (MODE == 2) { k = q & 7; m = q >> 3; }
            else { m = q & 127; k = q >> 7; }
            const int gm = m0 + m, gk = k0 + k;
            const bool va = gm < M && gk < K;
            const double* pa =
                va ? (MODE == 2 ? A + (long long)gm * lda + gk : A + (long long)gk * lda + gm) : A;
            cp_async8(&As[buf][k][m], pa, va);
            int nn, kk;
            if (MODE == 0) { nn = q & 127; kk = q >> 7; }
            else { kk = q & 7; nn = q >> 3; }
            const int gn = n0 + nn, gk2 = k0 + kk;
            const bool vb = gn < N && gk2 < K;
            const double* pb =
                vb ? (MODE == 0 ? B + (long long)gk2 * ldb + gn : B + (long long)gn * ldb + gk2)
                   : B;
            cp_async8(&Bs[buf][kk][nn], pb, vb);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int nk = (K + GBK - 1) / GBK;
    issue(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        const int cur = kt & 1;
        if (kt + 1 < nk) issue(cur ^ 1, (kt + 1) * GBK);
        else asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();
#pragma unroll
        for (int k = 0; k < GBK; ++k) {
            double a[8], b[8];
            const double2* ap = reinterpret_cast<const double2*>(&As[cur][k][ty * 4]);
            const double2* ap2 = reinterpret_cast<const double2*>(&As[cur][k][64 + ty * 4]);
            const double2* bp = reinterpret_cast<const double2*>(&Bs[cur][k][tx * 4]);
            const double2* bp2 = reinterpret_cast<const double2*>(&Bs[cur][k][64 + tx * 4]);
            const double2 a0 = ap[0], a1 = ap[1], a2 = ap2[0], a3 = ap2[1];
            const double2 b0 = bp[0], b1 = bp[1], b2 = bp2[0], b3 = bp2[1];
            a[0] = a0.x; a[1] = a0.y; a[2] = a1.x; a[3] = a1.y;
            a[4] = a2.x; a[5] = a2.y; a[6] = a3.x; a[7] = a3.y;
            b[0] = b0.x; b[1] = b0.y; b[2] = b1.x; b[3] = b1.y;
            b[4] = b2.x; b[5] = b2.y; b[6] = b3.x; b[7] = b3.y;
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int c = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
        if (c >= N) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int r = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
            if (r < M && (!TRI || r >= c)) C[(long long)c * ldc + r] -= acc[i][j];
        }
    }
}

template <int MODE, bool TRI>
void dgemm_launch(cudaStream_t s, int M, int N, int K, const double* A, long long lda,
                  const double* B, long long ldb, double* C, long long ldc)
{
    const int tm = (M + GBM - 1) / GBM, tn = (N + GBN - 1) / GBN;
    dgemm_sub_kernel<MODE, TRI><<<(unsigned)((long long)tm * tn), GTHR, 0, s>>>(
        M, N, K, A, lda, B, ldb, C, ldc, tm);
}

// 64x64x16 tiles, 4x4 outputs per thread, register-staged prefetch: the
// tall, narrow updates of the panels and TRSM recursions (more CTAs).
constexpr int SBM = 64, SBN = 64, SBK = 16, STHR = 256;

// MODE 0: C -= A B^T (A M x K, B N x K); 1: C -= A B (B K x N);
// 2: C -= A^T B (A stored K x M, B K x N).  TRI: only entries with row >= col
// (local to C) are written and tiles wholly above the diagonal are skipped.
template <int MODE, bool TRI>
__global__ void __launch_bounds__(STHR) dgemm_sub64_kernel(int M, int N, int K,
                                                         const double* __restrict__ A,
                                                         long long lda,
                                                         const double* __restrict__ B,
                                                         long long ldb, double* C, long long ldc,
                                                         int tiles_m)
{
    __shared__ double As[SBK][SBM + 1];
    __shared__ double Bs[SBK][SBN + 1];
    const int tile = blockIdx.x;
    const int m0 = (tile % tiles_m) * SBM, n0 = (tile / tiles_m) * SBN;
    if (TRI && n0 >= m0 + SBM) return;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    double ra[4], rb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int q = tid + e * STHR;
            int m, k;
            if (MODE == 2) { k = q & 15; m = q >> 4; }
            else { m = q & 63; k = q >> 6; }
            const int gm = m0 + m, gk = k0 + k;
            double v = 0.0;
            if (gm < M && gk < K)
                v = MODE == 2 ? A[(long long)gm * lda + gk] : A[(long long)gk * lda + gm];
            ra[e] = v;
            int nn, kk;
            if (MODE == 0) { nn = q & 63; kk = q >> 6; }
            else { kk = q & 15; nn = q >> 4; }
            const int gn = n0 + nn, gk2 = k0 + kk;
            double w = 0.0;
            if (gn < N && gk2 < K)
                w = MODE == 0 ? B[(long long)gk2 * ldb + gn] : B[(long long)gn * ldb + gk2];
            rb[e] = w;
        }
    };
    auto stash = [&]() {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int q = tid + e * STHR;
            if (MODE == 2) As[q & 15][q >> 4] = ra[e];
            else As[q >> 6][q & 63] = ra[e];
            if (MODE == 0) Bs[q >> 6][q & 63] = rb[e];
            else Bs[q & 15][q >> 4] = rb[e];
        }
    };
    const int nk = (K + SBK - 1) / SBK;
    fetch(0);
    for (int kt = 0; kt < nk; ++kt) {
        stash();
        __syncthreads();
        if (kt + 1 < nk) fetch((kt + 1) * SBK);
#pragma unroll
        for (int k = 0; k < SBK; ++k) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int c = n0 + tx + 16 * j;
        if (c >= N) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = m0 + ty + 16 * i;
            if (r < M && (!TRI || r >= c)) C[(long long)c * ldc + r] -= acc[i][j];
        }
    }
}

template <int MODE, bool TRI>
void dgemm_launch64(cudaStream_t s, int M, int N, int K, const double* A, long long lda,
                  const double* B, long long ldb, double* C, long long ldc)
{
    const int tm = (M + SBM - 1) / SBM, tn = (N + SBN - 1) / SBN;
    dgemm_sub64_kernel<MODE, TRI><<<(unsigned)((long long)tm * tn), STHR, 0, s>>>(
        M, N, K, A, lda, B, ldb, C, ldc, tm);
}

hdbf_status dgemm(hdbf_context* ctx, int mode, bool lower_only, int M, int N, int K,
                  const double* A, long long lda, const double* B, long long ldb, double* C,
                  long long ldc)
{
    if (M <= 0 || N <= 0 || K <= 0) return HDBF_STATUS_SUCCESS;
    if (!A || !B || !C) return HDBF_STATUS_INVALID_VALUE;
    if (lower_only && mode != 0) return HDBF_STATUS_INVALID_VALUE;
    const long long tiles = (long long)((M + SBM - 1) / SBM) * ((N + SBN - 1) / SBN);
    if (tiles > 0x7fffffffLL) return HDBF_STATUS_NOT_SUPPORTED;
    double flops = 2.0 * (double)M * N * K;
    if (lower_only) {
        const double d = (double)(M < N ? M : N);
        flops = 2.0 * (double)K * (d * (double)M - d * (d - 1.0) / 2.0);
    }
    ProfScope prof(ctx, kClsGemm, flops, 8.0 * ((double)M * K + (double)N * K + 2.0 * M * N), M,
                   N, K);
    cudaStream_t s = ctx->stream;
    // 128x128 tiles only when they still give two waves of CTAs (one per SM)
    const long long big_tiles = (long long)((M + GBM - 1) / GBM) * ((N + GBN - 1) / GBN);
    if (big_tiles >= 2LL * ctx->sm_count) {
        if (mode == 0) {
            if (lower_only) dgemm_launch<0, true>(s, M, N, K, A, lda, B, ldb, C, ldc);
            else dgemm_launch<0, false>(s, M, N, K, A, lda, B, ldb, C, ldc);
        } else if (mode == 1) {
            dgemm_launch<1, false>(s, M, N, K, A, lda, B, ldb, C, ldc);
        } else {
            dgemm_launch<2, false>(s, M, N, K, A, lda, B, ldb, C, ldc);
        }
    } else {
        if (mode == 0) {
            if (lower_only) dgemm_launch64<0, true>(s, M, N, K, A, lda, B, ldb, C, ldc);
            else dgemm_launch64<0, false>(s, M, N, K, A, lda, B, ldb, C, ldc);
        } else if (mode == 1) {
            dgemm_launch64<1, false>(s, M, N, K, A, lda, B, ldb, C, ldc);
        } else {
            dgemm_launch64<2, false>(s, M, N, K, A, lda, B, ldb, C, ldc);
        }
    }
    ctx->launches++;
    return last_cuda(ctx);
}

// ------------------------------------------------------------- potf2 leaf
// n <= 64 Cholesky of the lower triangle, one CTA; LAPACK xPOTRF pivot test
// and info as the FP32 leaf: the first column whose updated diagonal is not
// > 0 (or is NaN) stops the factorization with its value left in place and
// info = info_base + j + 1 (first failure wins); a block whose info is
// already non-zero is left untouched.
__global__ void __launch_bounds__(256) dpotf2_kernel(int n, double* A, long long lda, int* info,
                                                     int info_base)
{
    __shared__ double S[kL][kL + 1];  // S[c][r] = A(r, c)
    const int tid = threadIdx.x;
    if (info && *reinterpret_cast<volatile int*>(info) != 0) return;
    for (int q = tid; q < kL * kL; q += 256) {
        const int c = q >> 6, r = q & 63;
        S[c][r] = (r < n && c < n && r >= c) ? A[(long long)c * lda + r] : 0.0;
    }
    __syncthreads();
    int failed_at = -1;
    for (int j = 0; j < n; ++j) {
        const double d = S[j][j];
        if (!(d > 0.0)) {  // uniform: every thread read the same value
            failed_at = j;
            break;
        }
        const double sd = sqrt(d);
        const double rcp = 1.0 / sd;
        __syncthreads();
        if (tid == j) S[j][j] = sd;
        if (tid > j && tid < n) S[j][tid] *= rcp;
        __syncthreads();
        const int t = n - j - 1;
        for (int q = tid; q < t * t; q += 256) {
            const int c = j + 1 + q / t, r = j + 1 + q % t;
            if (r >= c) S[c][r] = fma(-S[j][r], S[j][c], S[c][r]);
        }
        __syncthreads();
    }
    __syncthreads();
    for (int q = tid; q < kL * kL; q += 256) {
        const int c = q >> 6, r = q & 63;
        if (r < n && c < n && r >= c) A[(long long)c * lda + r] = S[c][r];
    }
    if (failed_at >= 0 && tid == 0 && info) atomicCAS(info, 0, info_base + failed_at + 1);
}

// ------------------------------------------------------ triangular leaves
// Inverses of the 64x64 diagonal blocks of a lower-triangular matrix (unit
// or non-unit), one CTA per block, thread t solving L_bb x = e_t by forward
// substitution.  out[b*4096 + c*64 + r] = inv(L_bb)(r, c); a partial last
// block is padded with the identity.
__global__ void __launch_bounds__(kL) dtri_inv64_kernel(int n, const double* __restrict__ L,
                                                        long long ldl, int unit, double* out)
{
    __shared__ double Ls[kL][kL + 1];  // Ls[r][c] = L(base + r, base + c)
    const int base = blockIdx.x * kL;
    const int nb = min(kL, n - base);
    const int t = threadIdx.x;
    for (int idx = t; idx < kL * kL; idx += kL) {
        const int c = idx / kL, r = idx - c * kL;
        Ls[r][c] = (r < nb && c < nb && r >= c) ? L[(long long)(base + c) * ldl + base + r] : 0.0;
    }
    __syncthreads();
    double x[kL];
#pragma unroll
    for (int i = 0; i < kL; ++i) x[i] = (i == t) ? 1.0 : 0.0;
#pragma unroll
    for (int k = 0; k < kL; ++k) {
        if (k < nb) {
            if (!unit) x[k] = x[k] / Ls[k][k];
#pragma unroll
            for (int i = k + 1; i < kL; ++i) x[i] = fma(-Ls[i][k], x[k], x[i]);
        }
    }
    double* ob = out + (long long)blockIdx.x * kL * kL + (long long)t * kL;
#pragma unroll
    for (int i = 0; i < kL; ++i) ob[i] = x[i];
}

constexpr size_t kApplySmem = sizeof(double) * 2 * kL * (kL + 1);

// B(rows x cols) <- inv * B for rows <= 64: CTA = 64 columns of B, in place.
__global__ void __launch_bounds__(256) dllu_apply_kernel(int rows, int cols,
                                                         const double* __restrict__ inv,
                                                         double* B, long long ldb)
{
    extern __shared__ double dsm[];
    double* Is = dsm;                   // Is[k*65 + r] = inv(r, k)
    double* Bs = dsm + kL * (kL + 1);   // Bs[k*65 + c] = B(k, c0 + c)
    const int tid = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * kL;
    for (int idx = tid; idx < kL * kL; idx += 256) {
        const int k = idx >> 6, r = idx & 63;
        Is[k * (kL + 1) + r] = inv[idx];
        const int c = idx >> 6, kk = idx & 63;
        Bs[kk * (kL + 1) + c] = (kk < rows && c0 + c < cols) ? B[(c0 + c) * ldb + kk] : 0.0;
    }
    __syncthreads();
    const int ty = tid >> 4, tx = tid & 15;
    double acc[4][4] = {};
    for (int k = 0; k < kL; ++k) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = Is[k * (kL + 1) + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[k * (kL + 1) + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const long long c = c0 + tx + 16 * j;
        if (c >= cols) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = ty + 16 * i;
            if (r < rows) B[c * ldb + r] = acc[i][j];
        }
    }
}

// B(rows x cols) <- B * inv^T for cols <= 64: CTA = 64 rows of B, in place.
__global__ void __launch_bounds__(256) drlt_apply_kernel(int rows, int cols,
                                                         const double* __restrict__ inv,
                                                         double* B, long long ldb)
{
    extern __shared__ double dsm[];
    double* Bs = dsm;                   // Bs[k*65 + r] = B(r0 + r, k)
    double* Is = dsm + kL * (kL + 1);   // Is[k*65 + c] = inv(c, k)
    const int tid = threadIdx.x;
    const long long r0 = (long long)blockIdx.x * kL;
    for (int idx = tid; idx < kL * kL; idx += 256) {
        const int k = idx >> 6, x = idx & 63;
        Is[k * (kL + 1) + x] = inv[idx];
        Bs[k * (kL + 1) + x] = (k < cols && r0 + x < rows) ? B[(long long)k * ldb + r0 + x] : 0.0;
    }
    __syncthreads();
    const int ty = tid >> 4, tx = tid & 15;
    double acc[4][4] = {};
    for (int k = 0; k < kL; ++k) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = Bs[k * (kL + 1) + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Is[k * (kL + 1) + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int c = tx + 16 * j;
        if (c >= cols) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const long long r = r0 + ty + 16 * i;
            if (r < rows) B[(long long)c * ldb + r] = acc[i][j];
        }
    }
}

hdbf_status dtri_inv(hdbf_context* ctx, int n, const double* L, long long ldl, bool unit,
                     double* inv)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    const int nb = (n + kL - 1) / kL;
    ProfScope prof(ctx, kClsTrsmInv, (double)nb * kL * kL * kL / 3.0, 8.0 * 2.0 * nb * kL * kL);
    dtri_inv64_kernel<<<nb, kL, 0, ctx->stream>>>(n, L, ldl, unit ? 1 : 0, inv);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status dllu_apply(hdbf_context* ctx, int rows, int cols, const double* inv, double* B,
                       long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    ProfScope prof(ctx, kClsTrsmL, (double)rows * rows * cols, 16.0 * (double)rows * cols);
    const long long grid = ((long long)cols + kL - 1) / kL;
    dllu_apply_kernel<<<(unsigned)grid, 256, kApplySmem, ctx->stream>>>(rows, cols, inv, B, ldb);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status drlt_apply(hdbf_context* ctx, int rows, int cols, const double* inv, double* B,
                       long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    ProfScope prof(ctx, kClsTrsmR, (double)cols * cols * rows, 16.0 * (double)rows * cols);
    const long long grid = ((long long)rows + kL - 1) / kL;
    drlt_apply_kernel<<<(unsigned)grid, 256, kApplySmem, ctx->stream>>>(rows, cols, inv, B, ldb);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status trsm_rlt_rec64(hdbf_context* ctx, int rows, int cols, const double* L,
                           long long ldl, double* B, long long ldb, const double* inv)
{
    if (cols <= kL) return drlt_apply(ctx, rows, cols, inv, B, ldb);
    const int c1 = split64(cols);
    const int c2 = cols - c1;
    HDBF_TRY(trsm_rlt_rec64(ctx, rows, c1, L, ldl, B, ldb, inv));
    HDBF_TRY(dgemm(ctx, 0, false, rows, c2, c1, B, ldb, L + c1, ldl, B + (long long)c1 * ldb,
                   ldb));
    return trsm_rlt_rec64(ctx, rows, c2, L + (long long)c1 * ldl + c1, ldl,
                          B + (long long)c1 * ldb, ldb, inv + (long long)(c1 / kL) * kL * kL);
}

hdbf_status trsm_llu_rec64(hdbf_context* ctx, int rows, int cols, const double* L,
                           long long ldl, double* B, long long ldb, const double* inv)
{
    if (rows <= kL) return dllu_apply(ctx, rows, cols, inv, B, ldb);
    const int r1 = split64(rows);
    const int r2 = rows - r1;
    HDBF_TRY(trsm_llu_rec64(ctx, r1, cols, L, ldl, B, ldb, inv));
    HDBF_TRY(dgemm(ctx, 1, false, r2, cols, r1, L + r1, ldl, B, ldb, B + r1, ldb));
    return trsm_llu_rec64(ctx, r2, cols, L + (long long)r1 * ldl + r1, ldl, B + r1, ldb,
                          inv + (long long)(r1 / kL) * kL * kL);
}

// ------------------------------------------------------------ panel leaf
constexpr int kPThreads = 256;
constexpr int kPMaxW = 64;
constexpr int kPMaxGrid = 256;
// Slot in doubles: [seq (u32) | |a| | row (int) | pad | candidate row | diagonal row]
constexpr int kPSlot = 4 + 2 * kPMaxW;

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

__device__ __forceinline__ bool dbetter(double v, int i, double bv, int bi)
{
    if (i == INT_MAX) return false;
    if (bi == INT_MAX) return true;
    return v > bv || (v == bv && i < bi);
}

__global__ void __launch_bounds__(kPThreads)
getf2_coop64_kernel(int m, int w, double* A, long long lda, int rpc, int* ipiv, int ipiv_add,
                    int* info, int info_base, double* scr, unsigned* epoch_ptr,
                    unsigned* done_ptr, int* err, int pivot)
{
    extern __shared__ double dtile[];  // dtile[c * rpc + r]
    __shared__ double prow[kPMaxW];
    __shared__ double orow[kPMaxW];
    __shared__ double red_v[kPThreads / 32];
    __shared__ int red_i[kPThreads / 32];
    __shared__ double cv[kPMaxGrid];
    __shared__ int ci[kPMaxGrid];
    __shared__ int s_best_row, s_win_cta, s_abort, s_last;

    const int G = gridDim.x;
    const int cta = blockIdx.x;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int r0 = cta * rpc;
    const int nr = max(0, min(m, r0 + rpc) - r0);
    const unsigned epoch = *reinterpret_cast<volatile unsigned*>(epoch_ptr);
    auto slot_of = [&](int par, int q) { return scr + ((long long)par * kPMaxGrid + q) * kPSlot; };

    for (int e = tid; e < nr * w; e += kPThreads) {
        const int c = e / nr, r = e - c * nr;
        dtile[c * rpc + r] = A[(long long)c * lda + r0 + r];
    }
    if (tid == 0) s_abort = 0;
    __syncthreads();

    const int steps = min(m, w);
    for (int j = 0; j < steps; ++j) {
        const int par = j & 1;
        const unsigned seq = (epoch << 8) + (unsigned)j + 1u;
        double* slot = slot_of(par, cta);
        const int owner = j / rpc;

        // 1. local candidate over owned rows >= j
        double bv = -1.0;
        int bi = INT_MAX;
        if (pivot) {
            for (int r = tid; r < nr; r += kPThreads) {
                if (r0 + r >= j) {
                    const double v = fabs(dtile[j * rpc + r]);
                    if (bi == INT_MAX || v > bv) { bv = v; bi = r0 + r; }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, bv, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                if (dbetter(ov, oi, bv, bi)) { bv = ov; bi = oi; }
            }
            if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
            __syncthreads();
            if (tid == 0) {
                for (int q = 1; q < kPThreads / 32; ++q)
                    if (dbetter(red_v[q], red_i[q], bv, bi)) { bv = red_v[q]; bi = red_i[q]; }
                s_best_row = bi;
                red_v[0] = bv;
            }
            __syncthreads();
        }

        // 2. publish
        const int my_best = pivot ? s_best_row : INT_MAX;
        if (tid < w) {
            if (my_best != INT_MAX) slot[4 + tid] = dtile[tid * rpc + (my_best - r0)];
            if (cta == owner) slot[4 + kPMaxW + tid] = dtile[tid * rpc + (j - r0)];
        }
        if (tid == 0) {
            slot[1] = pivot ? red_v[0] : -1.0;
            reinterpret_cast<int*>(slot + 2)[0] = my_best;
        }
        __syncthreads();
        // The release store (after the barrier) orders every thread's slot
        // writes before the sequence number that other CTAs acquire.
        if (tid == 0) st_release_u32(reinterpret_cast<unsigned*>(slot), seq);

        // 3. poll every slot (thread q watches CTA q), bounded
        for (int q = tid; q < G; q += kPThreads) {
            const double* sq = slot_of(par, q);
            unsigned polls = 0;
            while (ld_acquire_u32(reinterpret_cast<const unsigned*>(sq)) != seq) {
                if (++polls > spin_limit_of(err)) {
                    atomicCAS(err, 0, kErrTimeout);
                    s_abort = 1;
                    break;
                }
                if (polls > 256) __nanosleep(32);
            }
            cv[q] = __ldcg(sq + 1);
            ci[q] = __ldcg(reinterpret_cast<const int*>(sq + 2));
        }
        __syncthreads();
        if (s_abort) break;

        // 4. global winner, identical on every CTA
        if (!pivot) {
            if (tid == 0) { s_best_row = j; s_win_cta = -1; }
        } else if (warp == 0) {
            double gv = -1.0;
            int gi = INT_MAX, gc = 0;
            for (int q = lane; q < G; q += 32)
                if (dbetter(cv[q], ci[q], gv, gi)) { gv = cv[q]; gi = ci[q]; gc = q; }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, gv, off);
                const int oi = __shfl_down_sync(0xffffffffu, gi, off);
                const int oc = __shfl_down_sync(0xffffffffu, gc, off);
                if (dbetter(ov, oi, gv, gi)) { gv = ov; gi = oi; gc = oc; }
            }
            if (lane == 0) { s_best_row = gi; s_win_cta = gc; }
        }
        __syncthreads();
        const int p = s_best_row;
        if (tid < w) {
            const double* so = slot_of(par, owner);
            orow[tid] = __ldcg(so + 4 + kPMaxW + tid);
            if (s_win_cta >= 0) prow[tid] = __ldcg(slot_of(par, s_win_cta) + 4 + tid);
            else prow[tid] = orow[tid];
        }
        if (pivot && cta == 0 && tid == 0) ipiv[j] = p + 1 + ipiv_add;
        __syncthreads();

        // 5. swap rows j and p (within this column block), scale, rank-1 update
        if (p != j && tid < w) {
            if (j >= r0 && j < r0 + nr) dtile[tid * rpc + (j - r0)] = prow[tid];
            if (p >= r0 && p < r0 + nr) dtile[tid * rpc + (p - r0)] = orow[tid];
        }
        __syncthreads();
        const double piv = prow[j];
        const bool nz = piv != 0.0;
        const bool recip = fabs(piv) >= DBL_MIN;
        const double rcp = 1.0 / piv;
        if (!nz && cta == 0 && tid == 0 && info) atomicCAS(info, 0, info_base + j + 1);
        for (int r = tid; r < nr; r += kPThreads) {
            if (r0 + r > j) {
                double l = dtile[j * rpc + r];
                if (nz) {
                    l = recip ? l * rcp : l / piv;
                    dtile[j * rpc + r] = l;
                }
                for (int c = j + 1; c < w; ++c)
                    dtile[c * rpc + r] = fma(-l, prow[c], dtile[c * rpc + r]);
            }
        }
        __syncthreads();
    }

    for (int e = tid; e < nr * w; e += kPThreads) {
        const int c = e / nr, r = e - c * nr;
        A[(long long)c * lda + r0 + r] = dtile[c * rpc + r];
    }

    // Advance the shared launch counter once every CTA is done.
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(done_ptr, 1u) + 1u == (unsigned)G;
    }
    __syncthreads();
    if (s_last && tid == 0) {
        __threadfence();
        atomicExch(done_ptr, 0u);
        atomicAdd(epoch_ptr, 1u);
    }
}

hdbf_status getf2_coop64(hdbf_context* ctx, int m, int w, double* A, long long lda, int* ipiv,
                         int ipiv_add, int* info, int info_base, bool pivot)
{
    int piv_flag = pivot ? 1 : 0;
    if (m <= 0 || w <= 0) return HDBF_STATUS_SUCCESS;
    if (w > kPMaxW) return HDBF_STATUS_INVALID_VALUE;
    const size_t smem_cap = ctx->max_smem_optin > 8192 ? ctx->max_smem_optin - 8192 : 40960;
    const size_t row_bytes = (size_t)w * sizeof(double);
    const long long fit_rows = (long long)(smem_cap / row_bytes);
    const int target = ctx->panel_rows > 0 ? ctx->panel_rows : 256;
    int G = (m + target - 1) / target;
    if (fit_rows > 0 && (m + fit_rows - 1) / fit_rows > G) G = (int)((m + fit_rows - 1) / fit_rows);
    if (G > ctx->sm_count) G = ctx->sm_count;
    if (G > kPMaxGrid) G = kPMaxGrid;
    if (G < 1) G = 1;
    int rpc = (m + G - 1) / G;
    size_t smem = (size_t)rpc * w * sizeof(double);
    if (smem > smem_cap) return HDBF_STATUS_NOT_SUPPORTED;
    double* scr = ws_coop64(ctx);
    unsigned* epoch = reinterpret_cast<unsigned*>(ctx->dev_small + kSmallEpoch);
    unsigned* done = reinterpret_cast<unsigned*>(ctx->dev_small + kSmallDone);
    int* err = ctx->dev_small + kSmallErr;
    ProfScope prof(ctx, kClsPanel, (double)m * w * w - (double)w * w * w / 3.0, 16.0 * m * w);
    void* args[] = {&m, &w, &A, &lda, &rpc, &ipiv, &ipiv_add, &info, &info_base,
                    &scr, &epoch, &done, &err, &piv_flag};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)getf2_coop64_kernel, dim3(G),
                                                dim3(kPThreads), args, smem, ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    return HDBF_STATUS_SUCCESS;
}

// --------------------------------------------------------------- row moves
// Gather every moved source row of nc columns into scratch, then scatter to
// the targets (sources and targets are the same row set).
__global__ void dgather_rows_kernel(const double* A, long long lda, int nc, const int* src,
                                    const int* count, int cap, double* temp)
{
    const int cnt = min(*count, cap);
    const long long total = (long long)nc * cnt;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e / cnt), q = (int)(e - (long long)c * cnt);
        temp[(long long)c * cap + q] = A[(long long)c * lda + src[q]];
    }
}

__global__ void dscatter_rows_kernel(double* A, long long lda, int nc, const int* tgt,
                                     const int* count, int cap, const double* temp)
{
    const int cnt = min(*count, cap);
    const long long total = (long long)nc * cnt;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(e / cnt), q = (int)(e - (long long)c * cnt);
        A[(long long)c * lda + tgt[q]] = temp[(long long)c * cap + q];
    }
}

}  // namespace

size_t getf2_coop64_scratch_bytes()
{
    return align_up((size_t)2 * kPMaxGrid * kPSlot * sizeof(double), 256);
}

void configure_fp64_kernels(hdbf_context* ctx)
{
    const size_t cap = ctx->max_smem_optin > 8192 ? ctx->max_smem_optin - 8192 : 40960;
    cudaFuncSetAttribute(dllu_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kApplySmem);
    cudaFuncSetAttribute(drlt_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kApplySmem);
    cudaFuncSetAttribute(getf2_coop64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)cap);
    cudaGetLastError();
}

hdbf_status gemm_sub(hdbf_context* ctx, bool nn, bool lower_only, int M, int N, int K,
                     const double* A, long long lda, const double* B, long long ldb, double* C,
                     long long ldc)
{
    return dgemm(ctx, nn ? 1 : 0, lower_only, M, N, K, A, lda, B, ldb, C, ldc);
}

hdbf_status gemm_sub_tn(hdbf_context* ctx, int M, int N, int K, const double* A, long long lda,
                        const double* B, long long ldb, double* C, long long ldc)
{
    return dgemm(ctx, 2, false, M, N, K, A, lda, B, ldb, C, ldc);
}

hdbf_status potf2_small(hdbf_context* ctx, int n, double* A, long long lda, int* info,
                        int info_base)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    if (n > kL) return HDBF_STATUS_INVALID_VALUE;
    ProfScope prof(ctx, kClsPotf2, (double)n * n * n / 3.0, 8.0 * n * n);
    dpotf2_kernel<<<1, 256, 0, ctx->stream>>>(n, A, lda, info, info_base);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status trsm_rlt(hdbf_context* ctx, int rows, int cols, const double* L, long long ldl,
                     double* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    HDBF_TRY(ensure_ws(ctx, ws_order<double>(cols)));
    double* inv = reinterpret_cast<double*>(ws_inv(ctx));
    HDBF_TRY(dtri_inv(ctx, cols, L, ldl, false, inv));
    return trsm_rlt_rec64(ctx, rows, cols, L, ldl, B, ldb, inv);
}

hdbf_status trsm_llu(hdbf_context* ctx, int rows, int cols, const double* L, long long ldl,
                     double* B, long long ldb)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    HDBF_TRY(ensure_ws(ctx, ws_order<double>(rows)));
    double* inv = reinterpret_cast<double*>(ws_inv(ctx));
    HDBF_TRY(dtri_inv(ctx, rows, L, ldl, true, inv));
    return trsm_llu_rec64(ctx, rows, cols, L, ldl, B, ldb, inv);
}

hdbf_status syrk_lower(hdbf_context* ctx, int n, int k, const double* A, long long lda,
                       double* C, long long ldc)
{
    return dgemm(ctx, 0, true, n, n, k, A, lda, A, lda, C, ldc);
}

hdbf_status potrf_diag(hdbf_context* ctx, int n, double* A, long long lda, int* info,
                       int info_base)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    if (n <= kL) return potf2_small(ctx, n, A, lda, info, info_base);
    const int n1 = split64(n);
    const int n2 = n - n1;
    double* A21 = A + n1;
    double* A22 = A + (long long)n1 * lda + n1;
    HDBF_TRY(potrf_diag(ctx, n1, A, lda, info, info_base));
    HDBF_TRY(trsm_rlt(ctx, n2, n1, A, lda, A21, lda));
    HDBF_TRY(syrk_lower(ctx, n2, n1, A21, lda, A22, lda));
    return potrf_diag(ctx, n2, A22, lda, info, info_base + n1);
}

hdbf_status apply_moves(hdbf_context* ctx, double* A, long long lda, int ncols, const int* src,
                        const int* tgt, const int* count, int max_moves, double* temp,
                        long long temp_cols)
{
    if (ncols <= 0 || max_moves <= 0) return HDBF_STATUS_SUCCESS;
    if (!temp || temp_cols <= 0) return HDBF_STATUS_INVALID_VALUE;
    ProfScope prof(ctx, kClsMoves, 0.0, 16.0 * (double)max_moves * ncols);
    for (long long c = 0; c < ncols; c += temp_cols) {
        const int nc = (int)((ncols - c) < temp_cols ? (ncols - c) : temp_cols);
        const long long total = (long long)nc * max_moves;
        const int grid = (int)((total + 255) / 256 < 65535 ? (total + 255) / 256 : 65535);
        dgather_rows_kernel<<<grid, 256, 0, ctx->stream>>>(A + c * lda, lda, nc, src, count,
                                                           max_moves, temp);
        dscatter_rows_kernel<<<grid, 256, 0, ctx->stream>>>(A + c * lda, lda, nc, tgt, count,
                                                            max_moves, temp);
        ctx->launches += 2;
    }
    return last_cuda(ctx);
}

// Recursive (Toledo/Gustavson) LU of an m x w FP64 panel down to 64-column
// leaves on the grid-wide kernel; ipiv receives (local row + 1 + ipiv_add).
hdbf_status getrf_panel(hdbf_context* ctx, int m, int w, double* A, long long lda, int* ipiv,
                        int ipiv_add, int* info, int info_base, bool pivot, const GetrfWs& ws)
{
    if (m <= 0 || w <= 0) return HDBF_STATUS_SUCCESS;
    if (w <= kPMaxW) return getf2_coop64(ctx, m, w, A, lda, ipiv, ipiv_add, info, info_base, pivot);
    double* temp = reinterpret_cast<double*>(ws.temp);
    const int w1 = split64(w);
    const int w2 = w - w1;
    HDBF_TRY(getrf_panel(ctx, m, w1, A, lda, ipiv, ipiv_add, info, info_base, pivot, ws));
    double* A12 = A + (long long)w1 * lda;
    if (pivot) {
        HDBF_TRY(compose_swaps(ctx, ipiv, w1, ipiv_add, m, ws.src, ws.tgt, ws.count, ws.gperm,
                               info));
        HDBF_TRY(apply_moves(ctx, A12, lda, w2, ws.src, ws.tgt, ws.count, std::min(m, 2 * w1),
                             temp, ws.temp_cols));
    }
    HDBF_TRY(trsm_llu(ctx, w1, w2, A, lda, A12, lda));
    HDBF_TRY(dgemm(ctx, 1, false, m - w1, w2, w1, A + w1, lda, A12, lda, A12 + w1, lda));
    HDBF_TRY(getrf_panel(ctx, m - w1, w2, A12 + w1, lda, pivot ? ipiv + w1 : nullptr,
                         ipiv_add + w1, info, info_base + w1, pivot, ws));
    if (pivot) {
        HDBF_TRY(compose_swaps(ctx, ipiv + w1, w2, ipiv_add + w1, m - w1, ws.src, ws.tgt,
                               ws.count, ws.gperm, info));
        HDBF_TRY(apply_moves(ctx, A + w1, lda, w1, ws.src, ws.tgt, ws.count,
                             std::min(m - w1, 2 * w2), temp, ws.temp_cols));
    }
    return HDBF_STATUS_SUCCESS;
}

}  // namespace hdbf
