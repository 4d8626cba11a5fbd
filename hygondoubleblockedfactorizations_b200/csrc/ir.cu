// FP64 iterative refinement around the low-precision factorizations.
//
// Only the refinement residual r = b - A x and the update x += d run in FP64
// on the GPU; the correction d = A^{-1} r is solved with the FP32 factors
// (after scaling each residual column by its infinity norm so that the FP32
// solve never underflows).  Not part of the reference, which has no solve.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"
#include "getrf/double_blocked_getrf.h"
#include "hdbf/mixed.h"
#include "potrf/double_blocked_potrf.h"

namespace hdbf {

hdbf_status potrf_mixed(hdbf_context* ctx, int prec, float* A, long long lda, int n, int b,
                        int* info);
hdbf_status getrf_mixed(hdbf_context* ctx, int prec, float* A, long long lda, int n, int b,
                        int* ipiv, int* info);
size_t mixed_shadow_bytes(int n, int b, bool split);

namespace {

constexpr int kRhsGroup = 16;
constexpr int kSplits = 16;
constexpr int kRowsPerCta = 256;
constexpr int kJChunk = 32;

__global__ void d2s_kernel(const double* __restrict__ A, long long lda, float* W, long long ldw,
                           int rows, int cols)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const long long c = blockIdx.y;
    if (r < rows && c < cols) W[c * ldw + r] = (float)A[c * lda + r];
}

// partial[s][c][r] = sum_{j in split s} A(r, j) * X(j, c) for the RHS group
// blockIdx.z (columns 16 z .. 16 z + 15).
__global__ void __launch_bounds__(kRowsPerCta) resid_partial_kernel(
    const double* __restrict__ A, long long lda, const double* __restrict__ X, long long ldx, int n,
    int nrhs, double* partial)
{
    __shared__ double xs[kJChunk][kRhsGroup];
    const int r = blockIdx.x * kRowsPerCta + threadIdx.x;
    const int s = blockIdx.y;
    const int c0 = blockIdx.z * kRhsGroup;
    const int nc = min(kRhsGroup, nrhs - c0);
    const int per = (n + kSplits - 1) / kSplits;
    const int j0 = s * per, j1 = min(n, j0 + per);
    double acc[kRhsGroup];
#pragma unroll
    for (int c = 0; c < kRhsGroup; ++c) acc[c] = 0.0;
    for (int jb = j0; jb < j1; jb += kJChunk) {
        const int jn = min(kJChunk, j1 - jb);
        __syncthreads();
        for (int idx = threadIdx.x; idx < kJChunk * kRhsGroup; idx += kRowsPerCta) {
            const int jj = idx / kRhsGroup, c = idx % kRhsGroup;
            xs[jj][c] = (jj < jn && c < nc) ? X[(long long)(c0 + c) * ldx + jb + jj] : 0.0;
        }
        __syncthreads();
        if (r < n) {
            for (int jj = 0; jj < jn; ++jj) {
                const double a = A[(long long)(jb + jj) * lda + r];
#pragma unroll
                for (int c = 0; c < kRhsGroup; ++c) acc[c] = fma(a, xs[jj][c], acc[c]);
            }
        }
    }
    if (r < n)
        for (int c = 0; c < nc; ++c)
            partial[((long long)s * nrhs + c0 + c) * n + r] = acc[c];
}

// R(r, c) = B(r, c) - sum_s partial[s][c][r]
__global__ void resid_final_kernel(const double* __restrict__ partial, const double* B,
                                   long long ldb, double* R, long long ldr, int n, int nrhs)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n || c >= nrhs) return;
    double acc = 0.0;
    for (int s = 0; s < kSplits; ++s) acc += partial[((long long)s * nrhs + c) * n + r];
    R[(long long)c * ldr + r] = B[(long long)c * ldb + r] - acc;
}

// out[c] = max_r |V(r, c)| (non-negative doubles order like their bits)
__global__ void colmax_kernel(const double* __restrict__ V, long long ldv, int n,
                              unsigned long long* out)
{
    const int c = blockIdx.y;
    double m = 0.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        m = fmax(m, fabs(V[(long long)c * ldv + r]));
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out + c, (unsigned long long)__double_as_longlong(m));
}

// rowsum partials for ||A||_inf: partial[s][r] = sum_{j in split s} |A(r, j)|
__global__ void rowabs_partial_kernel(const double* __restrict__ A, long long lda, int n,
                                      double* partial)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int s = blockIdx.y;
    if (r >= n) return;
    const int per = (n + kSplits - 1) / kSplits;
    const int j0 = s * per, j1 = min(n, j0 + per);
    double acc = 0.0;
    for (int j = j0; j < j1; ++j) acc += fabs(A[(long long)j * lda + r]);
    partial[(long long)s * n + r] = acc;
}

__global__ void rowabs_final_kernel(const double* __restrict__ partial, int n,
                                    unsigned long long* out)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    double v = 0.0;
    if (r < n)
        for (int s = 0; s < kSplits; ++s) v += partial[(long long)s * n + r];
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
}

// F(r, c) = (float)(V(r, c) / nrm[c])
__global__ void scale_to_f32_kernel(const double* __restrict__ V, long long ldv,
                                    const unsigned long long* nrm, float* F, long long ldf, int n,
                                    int nrhs)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n || c >= nrhs) return;
    const double s = __longlong_as_double((long long)nrm[c]);
    F[(long long)c * ldf + r] = s > 0.0 ? (float)(V[(long long)c * ldv + r] / s) : 0.f;
}

// X(r, c) (+)= (double)F(r, c) * nrm[c]
__global__ void update_x_kernel(const float* __restrict__ F, long long ldf,
                                const unsigned long long* nrm, double* X, long long ldx, int n,
                                int nrhs, int accumulate)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n || c >= nrhs) return;
    const double s = __longlong_as_double((long long)nrm[c]);
    const double d = (double)F[(long long)c * ldf + r] * s;
    double* x = X + (long long)c * ldx + r;
    *x = accumulate ? *x + d : d;
}

// ---- GMRES-IR kernels (FP64; vector block j of V at V + j * vstride, column c
// at + c * n)
constexpr int kDotChunks = 64;

// Y(r, c) = sum_s partial[s][c][r]  (the product A X of resid_partial_kernel)
__global__ void matvec_final_kernel(const double* __restrict__ partial, double* Y, int n, int nrhs)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n || c >= nrhs) return;
    double acc = 0.0;
    for (int s = 0; s < kSplits; ++s) acc += partial[((long long)s * nrhs + c) * n + r];
    Y[(long long)c * n + r] = acc;
}

// partial[(j * nrhs + c) * kDotChunks + chunk] = sum over the chunk's rows of
// V_j(r, c) * Wv(r, c); fixed-order tree reduction (deterministic).
__global__ void __launch_bounds__(256) dot_partial_kernel(const double* __restrict__ V,
                                                          long long vstride,
                                                          const double* __restrict__ Wv, int n,
                                                          int nrhs, double* partial)
{
    __shared__ double red[256];
    const int chunk = blockIdx.x, j = blockIdx.y, c = blockIdx.z;
    const int per = (n + kDotChunks - 1) / kDotChunks;
    const int r0 = chunk * per, r1 = min(n, r0 + per);
    const double* v = V + (long long)j * vstride + (long long)c * n;
    const double* w = Wv + (long long)c * n;
    double acc = 0.0;
    for (int r = r0 + threadIdx.x; r < r1; r += 256) acc = fma(v[r], w[r], acc);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] += red[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[((long long)j * nrhs + c) * kDotChunks + chunk] = red[0];
}

// H[j * nrhs + c] = sum over chunks (in order)
__global__ void dot_final_kernel(const double* __restrict__ partial, int nj, int nrhs, double* H)
{
    const int t = blockIdx.x * 256 + threadIdx.x;
    if (t >= nj * nrhs) return;
    double acc = 0.0;
    for (int q = 0; q < kDotChunks; ++q) acc += partial[(long long)t * kDotChunks + q];
    H[t] = acc;
}

// Wv(r, c) -= sum_{j < nj} V_j(r, c) H[j * nrhs + c]
__global__ void axpy_kernel(const double* __restrict__ V, long long vstride, int nj,
                            const double* __restrict__ H, double* Wv, int n, int nrhs)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n || c >= nrhs) return;
    double acc = Wv[(long long)c * n + r];
    for (int j = 0; j < nj; ++j)
        acc = fma(-V[(long long)j * vstride + (long long)c * n + r], H[j * nrhs + c], acc);
    Wv[(long long)c * n + r] = acc;
}

// Vout(r, c) = Wv(r, c) / sqrt(sq[c])  (0 when sq[c] == 0)
__global__ void normalize_kernel(const double* __restrict__ Wv, const double* __restrict__ sq,
                                 double* Vout, int n, int nrhs)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n || c >= nrhs) return;
    const double nr = sqrt(sq[c]);
    Vout[(long long)c * n + r] = nr > 0.0 ? Wv[(long long)c * n + r] / nr : 0.0;
}

// X(r, c) += sum_{j < nj} V_j(r, c) Y[j * nrhs + c]
__global__ void combine_kernel(const double* __restrict__ V, long long vstride, int nj,
                               const double* __restrict__ Y, double* X, long long ldx, int n,
                               int nrhs)
{
    const int r = blockIdx.x * 256 + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n || c >= nrhs) return;
    double acc = 0.0;
    for (int j = 0; j < nj; ++j)
        acc = fma(V[(long long)j * vstride + (long long)c * n + r], Y[j * nrhs + c], acc);
    X[(long long)c * ldx + r] += acc;
}

struct IrBuffers {
    float* W = nullptr;      // FP32 working copy / factors (n x n, ld n)
    int* ipiv = nullptr;
    int* perm = nullptr;
    int* info = nullptr;
    double* R = nullptr;     // n x nrhs residual
    float* F = nullptr;      // n x nrhs scaled FP32 right-hand side / correction
    float* F2 = nullptr;     // permuted copy for GETRS
    double* part = nullptr;  // kSplits x nrhs x n partial sums
    unsigned long long* nrm = nullptr;  // [0, nrhs): column norms; [nrhs]: ||A||_inf
    // GMRES-IR (present when m > 0): Krylov basis, A v, dot partials, the
    // Hessenberg column (h, h2, ||w||^2) and the least-squares solution.
    int m = 0;
    double* V = nullptr;     // (m + 1) blocks of n x nrhs
    double* T = nullptr;     // n x nrhs
    double* dpart = nullptr; // kDotChunks x (m + 1) x nrhs
    double* Hd = nullptr;    // 2 (m + 1) nrhs + nrhs doubles
    double* Yd = nullptr;    // (m + 1) x nrhs
};

inline size_t al(size_t x) { return (x + 255) / 256 * 256; }

size_t ir_bytes(int n, int nrhs, int m = 0)
{
    size_t b = al((size_t)n * n * 4) + 3 * al((size_t)n * 4) + al(64) + al((size_t)n * nrhs * 8) +
               2 * al((size_t)n * nrhs * 4) + al((size_t)kSplits * nrhs * n * 8) +
               al((size_t)(nrhs + 1) * 8) + 4096;
    if (m > 0)
        b += al((size_t)(m + 1) * n * nrhs * 8) + al((size_t)n * nrhs * 8) +
             al((size_t)kDotChunks * (m + 1) * nrhs * 8) + al((size_t)(2 * (m + 1) + 1) * nrhs * 8) +
             al((size_t)(m + 1) * nrhs * 8);
    return b;
}

IrBuffers carve(char* base, int n, int nrhs, int m = 0)
{
    IrBuffers b;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base + off;
        off += al(bytes);
        return p;
    };
    b.W = reinterpret_cast<float*>(take((size_t)n * n * 4));
    b.ipiv = reinterpret_cast<int*>(take((size_t)n * 4));
    b.perm = reinterpret_cast<int*>(take((size_t)n * 4));
    take((size_t)n * 4);
    b.info = reinterpret_cast<int*>(take(64));
    b.R = reinterpret_cast<double*>(take((size_t)n * nrhs * 8));
    b.F = reinterpret_cast<float*>(take((size_t)n * nrhs * 4));
    b.F2 = reinterpret_cast<float*>(take((size_t)n * nrhs * 4));
    b.part = reinterpret_cast<double*>(take((size_t)kSplits * nrhs * n * 8));
    b.nrm = reinterpret_cast<unsigned long long*>(take((size_t)(nrhs + 1) * 8));
    if (m > 0) {
        b.m = m;
        b.V = reinterpret_cast<double*>(take((size_t)(m + 1) * n * nrhs * 8));
        b.T = reinterpret_cast<double*>(take((size_t)n * nrhs * 8));
        b.dpart = reinterpret_cast<double*>(take((size_t)kDotChunks * (m + 1) * nrhs * 8));
        b.Hd = reinterpret_cast<double*>(take((size_t)(2 * (m + 1) + 1) * nrhs * 8));
        b.Yd = reinterpret_cast<double*>(take((size_t)(m + 1) * nrhs * 8));
    }
    return b;
}

int next_precision(int prec)
{
    switch (prec) {
    case HDBF_PREC_BF16: return HDBF_PREC_BF16X3;
    case HDBF_PREC_FP16: return HDBF_PREC_FP16X3;
    case HDBF_PREC_BF16X3:
    case HDBF_PREC_FP16X3: return HDBF_PREC_FP32;
    default: return -1;
    }
}

// The adaptive driver's escalation: as next_precision, except that an LU
// factored with BF16 updates goes to the FP16 split (22 significant bits
// against BF16x3's 16, at the same cost; |L| <= 1 under partial pivoting and
// U's shadow carries a per-panel power-of-two scale, so FP16 covers the range)
int adaptive_next(bool spd, int prec)
{
    if (!spd && prec == HDBF_PREC_BF16) return HDBF_PREC_FP16X3;
    return next_precision(prec);
}

// Block sizes of the refinement's factorization: the fastest candidates of
// the exhaustive B200 sweep over n = 1024..32768 (the selector's training
// records).  FP32 POTRF: (2048, 256) below n = 16384, else (4096, 512).
// FP32 GETRF: (8192, 1024).  Mixed panel width: 256 below n = 12288, then
// 512, and 1024 from n = 16384 (GETRF) or n = 28672 (POTRF).
struct IrBlocks {
    int outer, inner;
};
IrBlocks ir_blocks(bool spd, int prec, int n)
{
    if (prec == HDBF_PREC_FP32) {
        if (spd) return n < 16384 ? IrBlocks{2048, 256} : IrBlocks{4096, 512};
        return IrBlocks{8192, 1024};
    }
    const int wide = spd ? 28672 : 16384;
    const int nb = n < 12288 ? 256 : (n < wide ? 512 : 1024);
    return IrBlocks{nb, nb};
}

class IrSolver {
public:
    IrSolver(hdbf_context* ctx, bool spd, const double* A, long long lda, int n, int nrhs,
             const double* B, long long ldb, double* X, long long ldx, const IrBuffers& buf)
        : ctx_(ctx), spd_(spd), A_(A), lda_(lda), n_(n), nrhs_(nrhs), B_(B), ldb_(ldb), X_(X),
          ldx_(ldx), b_(buf) {}

    hdbf_status factor(int prec, int* host_info)
    {
        cudaStream_t s = ctx_->stream;
        dim3 g((n_ + 255) / 256, n_);
        d2s_kernel<<<g, 256, 0, s>>>(A_, lda_, b_.W, n_, n_, n_);
        ctx_->launches++;
        HDBF_TRY(last_cuda(ctx_));
        const IrBlocks blk = ir_blocks(spd_, prec, n_);
        if (prec == HDBF_PREC_FP32) {
            if (spd_)
                double_blocked_potrf_kblocked_syrk(ctx_, b_.W, n_, n_, blk.outer, blk.inner, 0,
                                                   b_.info);
            else
                double_blocked_getrf(ctx_, b_.W, n_, n_, blk.outer, blk.inner,
                                     getrf_outer_trsm_direct, 0, b_.ipiv, b_.info);
            HDBF_TRY(ctx_->last_status);
        } else if (spd_) {
            HDBF_TRY(potrf_mixed(ctx_, prec, b_.W, n_, n_, blk.inner, b_.info));
        } else {
            HDBF_TRY(getrf_mixed(ctx_, prec, b_.W, n_, n_, blk.inner, b_.ipiv, b_.info));
        }
        if (!spd_) HDBF_TRY(ipiv_to_perm(ctx_, b_.ipiv, n_, b_.perm));
        if (cudaMemcpyAsync(host_info, b_.info, sizeof(int), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            cudaGetLastError();
            return HDBF_STATUS_CUDA_ERROR;
        }
        fallbacks_ = 0;
        if (spd_ && prec != HDBF_PREC_FP32) HDBF_TRY(hdbf_mixed_fallback_panels(ctx_, &fallbacks_));
        return HDBF_STATUS_SUCCESS;
    }
    // Cholesky panels the last factorization rebuilt in FP32 (panel fallback).
    int fallbacks() const { return fallbacks_; }

    // d = A^{-1} v with the FP32 factors; v scaled column-wise by nrm.
    hdbf_status correction(const double* V, long long ldv, bool accumulate)
    {
        return precond(V, ldv, X_, ldx_, accumulate);
    }

    // Out (+)= M^{-1} V, M the low-precision factorization (FP32 solves of the
    // column-scaled V).
    hdbf_status precond(const double* V, long long ldv, double* Out, long long ldo, bool accumulate)
    {
        cudaStream_t s = ctx_->stream;
        HDBF_TRY(colmax(V, ldv, b_.nrm));
        dim3 g((n_ + 255) / 256, nrhs_);
        scale_to_f32_kernel<<<g, 256, 0, s>>>(V, ldv, b_.nrm, b_.F, n_, n_, nrhs_);
        ctx_->launches++;
        float* sol = b_.F;
        if (spd_) {
            HDBF_TRY(potrs_f32(ctx_, b_.W, n_, n_, nrhs_, b_.F, n_));
        } else {
            HDBF_TRY(gather_rows_perm(ctx_, b_.F, n_, b_.F2, n_, b_.perm, n_, nrhs_));
            HDBF_TRY(getrs_f32_permuted(ctx_, b_.W, n_, n_, nrhs_, b_.F2, n_));
            sol = b_.F2;
        }
        update_x_kernel<<<g, 256, 0, s>>>(sol, n_, b_.nrm, Out, ldo, n_, nrhs_, accumulate ? 1 : 0);
        ctx_->launches++;
        return last_cuda(ctx_);
    }

    // Y = A X (FP64, X and Y n x nrhs with leading dimension n)
    hdbf_status matvec(const double* Xv, double* Y)
    {
        cudaStream_t s = ctx_->stream;
        dim3 g1((n_ + kRowsPerCta - 1) / kRowsPerCta, kSplits, (nrhs_ + kRhsGroup - 1) / kRhsGroup);
        ProfScope prof(ctx_, kClsIr, 2.0 * (double)n_ * n_ * nrhs_, 8.0 * (double)n_ * n_);
        resid_partial_kernel<<<g1, kRowsPerCta, 0, s>>>(A_, lda_, Xv, n_, n_, nrhs_, b_.part);
        dim3 g2((n_ + 255) / 256, nrhs_);
        matvec_final_kernel<<<g2, 256, 0, s>>>(b_.part, Y, n_, nrhs_);
        ctx_->launches += 2;
        return last_cuda(ctx_);
    }

    // H[j * nrhs + c] = <V_j(:, c), Wv(:, c)> for j < nj
    hdbf_status dots(const double* V, int nj, const double* Wv, double* H)
    {
        cudaStream_t s = ctx_->stream;
        const long long vs = (long long)n_ * nrhs_;
        dim3 g(kDotChunks, nj, nrhs_);
        dot_partial_kernel<<<g, 256, 0, s>>>(V, vs, Wv, n_, nrhs_, b_.dpart);
        dot_final_kernel<<<(nj * nrhs_ + 255) / 256, 256, 0, s>>>(b_.dpart, nj, nrhs_, H);
        ctx_->launches += 2;
        return last_cuda(ctx_);
    }

    hdbf_status axpy(const double* V, int nj, const double* H, double* Wv)
    {
        dim3 g((n_ + 255) / 256, nrhs_);
        axpy_kernel<<<g, 256, 0, ctx_->stream>>>(V, (long long)n_ * nrhs_, nj, H, Wv, n_, nrhs_);
        ctx_->launches++;
        return last_cuda(ctx_);
    }

    hdbf_status normalize(const double* Wv, const double* sq, double* Vout)
    {
        dim3 g((n_ + 255) / 256, nrhs_);
        normalize_kernel<<<g, 256, 0, ctx_->stream>>>(Wv, sq, Vout, n_, nrhs_);
        ctx_->launches++;
        return last_cuda(ctx_);
    }

    hdbf_status combine(const double* V, int nj, const double* Y)
    {
        dim3 g((n_ + 255) / 256, nrhs_);
        combine_kernel<<<g, 256, 0, ctx_->stream>>>(V, (long long)n_ * nrhs_, nj, Y, X_, ldx_, n_,
                                                    nrhs_);
        ctx_->launches++;
        return last_cuda(ctx_);
    }

    hdbf_status residual()
    {
        cudaStream_t s = ctx_->stream;
        dim3 g1((n_ + kRowsPerCta - 1) / kRowsPerCta, kSplits, (nrhs_ + kRhsGroup - 1) / kRhsGroup);
        ProfScope prof(ctx_, kClsIr, 2.0 * (double)n_ * n_ * nrhs_, 8.0 * (double)n_ * n_);
        resid_partial_kernel<<<g1, kRowsPerCta, 0, s>>>(A_, lda_, X_, ldx_, n_, nrhs_, b_.part);
        dim3 g2((n_ + 255) / 256, nrhs_);
        resid_final_kernel<<<g2, 256, 0, s>>>(b_.part, B_, ldb_, b_.R, n_, n_, nrhs_);
        ctx_->launches += 2;
        return last_cuda(ctx_);
    }

    hdbf_status colmax(const double* V, long long ldv, unsigned long long* out)
    {
        cudaMemsetAsync(out, 0, (size_t)nrhs_ * 8, ctx_->stream);
        dim3 g(64, nrhs_);
        colmax_kernel<<<g, 256, 0, ctx_->stream>>>(V, ldv, n_, out);
        ctx_->launches++;
        return last_cuda(ctx_);
    }

    hdbf_status host_colmax(const double* V, long long ldv, double* out)
    {
        HDBF_TRY(colmax(V, ldv, b_.nrm));
        if (cudaMemcpyAsync(out, b_.nrm, (size_t)nrhs_ * 8, cudaMemcpyDeviceToHost,
                            ctx_->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx_->stream) != cudaSuccess) {
            cudaGetLastError();
            return HDBF_STATUS_CUDA_ERROR;
        }
        return HDBF_STATUS_SUCCESS;
    }

    hdbf_status anorm(double* out)
    {
        dim3 g((n_ + 255) / 256, kSplits);
        rowabs_partial_kernel<<<g, 256, 0, ctx_->stream>>>(A_, lda_, n_, b_.part);
        cudaMemsetAsync(b_.nrm + nrhs_, 0, 8, ctx_->stream);
        rowabs_final_kernel<<<(n_ + 255) / 256, 256, 0, ctx_->stream>>>(b_.part, n_,
                                                                          b_.nrm + nrhs_);
        ctx_->launches += 2;
        unsigned long long bits = 0;
        if (cudaMemcpyAsync(&bits, b_.nrm + nrhs_, 8, cudaMemcpyDeviceToHost, ctx_->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(ctx_->stream) != cudaSuccess) {
            cudaGetLastError();
            return HDBF_STATUS_CUDA_ERROR;
        }
        memcpy(out, &bits, 8);
        return HDBF_STATUS_SUCCESS;
    }

    const IrBuffers& buffers() const { return b_; }

private:
    hdbf_context* ctx_;
    bool spd_;
    const double* A_;
    long long lda_;
    int n_, nrhs_;
    int fallbacks_ = 0;
    const double* B_;
    long long ldb_;
    double* X_;
    long long ldx_;
    IrBuffers b_;
};

hdbf_status xsv_mixed(hdbf_context* ctx, bool spd, int prec, int escalate, const double* A,
                      int lda, int n, int nrhs, const double* B, int ldb, double* X, int ldx,
                      double tol, int max_iter, hdbf_ir_info* out)
{
    hdbf_ir_info info;
    memset(&info, 0, sizeof(info));
    if (n < 0 || nrhs < 0 || nrhs > 64) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0 || nrhs == 0) {
        info.converged = 1;
        if (out) *out = info;
        return HDBF_STATUS_SUCCESS;
    }
    if (!A || !B || !X || lda < n || ldb < n || ldx < n) return HDBF_STATUS_INVALID_VALUE;
    if (prec < HDBF_PREC_FP32 || prec > HDBF_PREC_FP16X3) return HDBF_STATUS_INVALID_VALUE;
    if (max_iter < 0) max_iter = 0;
    HDBF_TRY(ensure_ws(ctx, n));
    // One arena for the shadows (offset 0) and the refinement buffers.
    const size_t shadow = mixed_shadow_bytes(n, 1024, true);  // widest panel ir_blocks picks
    hdbf_status st;
    char* arena = static_cast<char*>(mixed_arena(ctx, shadow + ir_bytes(n, nrhs), &st));
    if (!arena) return st;
    IrSolver solver(ctx, spd, A, lda, n, nrhs, B, ldb, X, ldx,
                    carve(arena + al(shadow), n, nrhs));

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timed = [&](double* acc, auto&& fn) -> hdbf_status {
        cudaEventRecord(e0, ctx->stream);
        const hdbf_status s2 = fn();
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        *acc += ms;
        return s2;
    };

    double anorm = 0.0;
    std::vector<double> bnorm(nrhs), rnorm(nrhs), xnorm(nrhs);
    st = solver.anorm(&anorm);
    if (st == HDBF_STATUS_SUCCESS) st = solver.host_colmax(B, ldb, bnorm.data());
    int cur = prec;
    if (st == HDBF_STATUS_SUCCESS) {
        int hinfo = 0;
        st = timed(&info.factor_ms, [&] { return solver.factor(cur, &hinfo); });
        info.factorizations = 1;
        while (st == HDBF_STATUS_SUCCESS && hinfo != 0 && escalate && next_precision(cur) >= 0) {
            // the panel fallback could not save it: refactor at the next precision
            cur = next_precision(cur);
            st = timed(&info.factor_ms, [&] { return solver.factor(cur, &hinfo); });
            info.factorizations++;
        }
        info.info = hinfo;
        info.fallback_panels = solver.fallbacks();
        if (st == HDBF_STATUS_SUCCESS && hinfo == 0)
            st = timed(&info.refine_ms, [&] { return solver.correction(B, ldb, false); });
        double prev = INFINITY;
        int stalls = 0;
        bool refactored = false;
        for (int it = 0; st == HDBF_STATUS_SUCCESS && hinfo == 0; ++it) {
            st = timed(&info.refine_ms, [&] { return solver.residual(); });
            if (st != HDBF_STATUS_SUCCESS) break;
            st = solver.host_colmax(solver.buffers().R, n, rnorm.data());
            if (st == HDBF_STATUS_SUCCESS) st = solver.host_colmax(X, ldx, xnorm.data());
            if (st != HDBF_STATUS_SUCCESS) break;
            double berr = 0.0;
            for (int c = 0; c < nrhs; ++c) {
                const double den = anorm * xnorm[c] + bnorm[c];
                const double e = den > 0.0 ? rnorm[c] / den : (rnorm[c] > 0.0 ? INFINITY : 0.0);
                berr = std::max(berr, std::isfinite(e) ? e : INFINITY);
            }
            if (it < HDBF_IR_HISTORY) info.history[it] = berr;
            info.backward_error = berr;
            info.iterations = it;
            if (berr <= tol) {
                info.converged = 1;
                break;
            }
            if (it >= max_iter) break;
            if (!(berr < 0.5 * prev)) {
                if (escalate && next_precision(cur) >= 0) {
                    cur = next_precision(cur);
                    int hinfo2 = 0;
                    st = timed(&info.factor_ms, [&] { return solver.factor(cur, &hinfo2); });
                    info.factorizations++;
                    info.info = hinfo2;
                    info.fallback_panels = solver.fallbacks();
                    if (hinfo2 != 0) break;
                    stalls = 0;
                    // the first correction with the new factors is not
                    // judged: forward error that the old factors left along
                    // the smallest singular directions shows up in the
                    // backward error only after it has been spread out
                    refactored = true;
                } else if (++stalls >= 2) {
                    break;
                }
            }
            prev = refactored ? INFINITY : std::min(prev, berr);
            refactored = false;
            st = timed(&info.refine_ms, [&] { return solver.correction(solver.buffers().R, n, true); });
        }
    }
    info.final_precision = cur;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (out) *out = info;
    return st;
}

// GMRES-IR: x0 = M^{-1} b; per outer step r = b - A x (FP64), then restarted
// left-preconditioned GMRES on M^{-1} A d = M^{-1} r (FP64 vectors, CGS2,
// Givens least squares on the host per right-hand side), x += d.
// Adaptive mode (`adaptive`): classical corrections d = M^{-1} r while each
// one at least halves the backward error; from the first that does not,
// GMRES steps on the same factors; when a GMRES step does not halve the
// backward error, or its rate would need more time than two factorizations
// to reach tol, the factorization is redone at the next precision (BF16 -> BF16x3 -> FP32,
// FP16 -> FP16x3 -> FP32) and classical corrections with the new factors
// continue from the current x, again until they stall.
// A general matrix factored with single-word BF16/FP16 updates skips the
// GMRES stage: its stalled classical corrections lead straight to the split
// (x3) factorization.
hdbf_status gmres_mixed(hdbf_context* ctx, bool spd, int prec, const double* A, int lda, int n,
                        int nrhs, const double* B, int ldb, double* X, int ldx, double tol,
                        int max_iter, int max_inner, double inner_tol, hdbf_ir_info* out,
                        bool adaptive = false)
{
    hdbf_ir_info info;
    memset(&info, 0, sizeof(info));
    if (n < 0 || nrhs < 0 || nrhs > 64) return HDBF_STATUS_INVALID_VALUE;
    if (n == 0 || nrhs == 0) {
        info.converged = 1;
        if (out) *out = info;
        return HDBF_STATUS_SUCCESS;
    }
    if (!A || !B || !X || lda < n || ldb < n || ldx < n) return HDBF_STATUS_INVALID_VALUE;
    if (prec < HDBF_PREC_FP32 || prec > HDBF_PREC_FP16X3) return HDBF_STATUS_INVALID_VALUE;
    if (max_iter < 0) max_iter = 0;
    const int m = max_inner <= 0 ? 30 : std::min(max_inner, 60);
    if (!(inner_tol > 0.0)) inner_tol = 1e-4;
    HDBF_TRY(ensure_ws(ctx, n));
    const size_t shadow = mixed_shadow_bytes(n, 1024, true);
    hdbf_status st;
    char* arena = static_cast<char*>(mixed_arena(ctx, shadow + ir_bytes(n, nrhs, m), &st));
    if (!arena) return st;
    const IrBuffers buf = carve(arena + al(shadow), n, nrhs, m);
    IrSolver solver(ctx, spd, A, lda, n, nrhs, B, ldb, X, ldx, buf);
    cudaStream_t strm = ctx->stream;

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timed = [&](double* acc, auto&& fn) -> hdbf_status {
        cudaEventRecord(e0, strm);
        const hdbf_status s2 = fn();
        cudaEventRecord(e1, strm);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        *acc += ms;
        return s2;
    };
    auto to_host = [&](void* dst, const void* src, size_t bytes) -> hdbf_status {
        if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, strm) != cudaSuccess ||
            cudaStreamSynchronize(strm) != cudaSuccess) {
            cudaGetLastError();
            return HDBF_STATUS_CUDA_ERROR;
        }
        return HDBF_STATUS_SUCCESS;
    };

    const long long vs = (long long)n * nrhs;
    double* h1 = buf.Hd;
    double* h2 = buf.Hd + (size_t)(m + 1) * nrhs;
    double* sq = buf.Hd + (size_t)2 * (m + 1) * nrhs;
    const size_t hbytes = (size_t)(2 * (m + 1) + 1) * nrhs * 8;
    std::vector<double> hh((size_t)(2 * (m + 1) + 1) * nrhs);
    std::vector<double> R((size_t)nrhs * (m + 1) * m, 0.0), g((size_t)nrhs * (m + 1), 0.0),
        cs((size_t)nrhs * m, 0.0), sn((size_t)nrhs * m, 0.0), beta(nrhs, 0.0),
        y((size_t)(m + 1) * nrhs, 0.0);
    double anorm = 0.0;
    std::vector<double> bnorm(nrhs), rnorm(nrhs), xnorm(nrhs);
    st = solver.anorm(&anorm);
    if (st == HDBF_STATUS_SUCCESS) st = solver.host_colmax(B, ldb, bnorm.data());
    int hinfo = 0;
    if (st == HDBF_STATUS_SUCCESS) {
        st = timed(&info.factor_ms, [&] { return solver.factor(prec, &hinfo); });
        info.factorizations = 1;
        info.info = hinfo;
        info.fallback_panels = solver.fallbacks();
    }
    int cur = prec;
    if (adaptive) {
        while (st == HDBF_STATUS_SUCCESS && hinfo != 0 && adaptive_next(spd, cur) >= 0) {
            // the panel fallback could not save it: refactor at the next precision
            cur = adaptive_next(spd, cur);
            st = timed(&info.factor_ms, [&] { return solver.factor(cur, &hinfo); });
            info.factorizations++;
            info.info = hinfo;
            info.fallback_panels = solver.fallbacks();
        }
    }
    // device time of the latest factorization and of the latest GMRES outer
    // step (residual + inner iterations): the escalation test weighs them
    double last_factor_ms = info.factorizations > 0 ? info.factor_ms / info.factorizations : 0.0;
    double last_step_ms = 0.0;
    if (st == HDBF_STATUS_SUCCESS && hinfo == 0)
        st = timed(&info.refine_ms, [&] { return solver.correction(B, ldb, false); });
    bool classical = adaptive;
    double prev = INFINITY;
    for (int it = 0; st == HDBF_STATUS_SUCCESS && hinfo == 0; ++it) {
        const double step_start = info.refine_ms;
        st = timed(&info.refine_ms, [&] { return solver.residual(); });
        if (st != HDBF_STATUS_SUCCESS) break;
        st = solver.host_colmax(buf.R, n, rnorm.data());
        if (st == HDBF_STATUS_SUCCESS) st = solver.host_colmax(X, ldx, xnorm.data());
        if (st != HDBF_STATUS_SUCCESS) break;
        double berr = 0.0;
        for (int c = 0; c < nrhs; ++c) {
            const double den = anorm * xnorm[c] + bnorm[c];
            const double e = den > 0.0 ? rnorm[c] / den : (rnorm[c] > 0.0 ? INFINITY : 0.0);
            berr = std::max(berr, std::isfinite(e) ? e : INFINITY);
        }
        if (it < HDBF_IR_HISTORY) info.history[it] = berr;
        info.backward_error = berr;
        info.iterations = it;
        if (berr <= tol) {
            info.converged = 1;
            break;
        }
        if (it >= max_iter) break;
        bool refactor = false;
        if (classical) {
            if (berr < 0.5 * prev) {
                prev = berr;
                st = timed(&info.refine_ms,
                           [&] { return solver.correction(buf.R, n, true); });
                continue;
            }
            classical = false;  // stalled: GMRES on the same factors from here
            // except on a single-word 16-bit LU, whose error grows with sqrt(n)
            // and the pivot growth: restarted GMRES (30 steps) on such factors
            // stalled at n = 32768 (BF16 at kappa 1e2, FP16 at kappa 1e4), so
            // refactor with the split operands at once
            refactor = !spd && (cur == HDBF_PREC_BF16 || cur == HDBF_PREC_FP16);
        } else if (adaptive) {
            // after a GMRES step: refactor when it did not halve the backward
            // error, or when the steps still needed at its rate would take
            // longer than two factorizations at the current precision (the
            // next precision's factorization costs 1.1x to 2.3x the current
            // one on B200)
            const double rate = berr / prev;
            if (!(rate < 0.5)) {
                refactor = true;
            } else {
                const double need = std::ceil(std::log(tol / berr) / std::log(rate));
                refactor = need * last_step_ms > 2.0 * last_factor_ms;
            }
        }
        if (refactor && adaptive_next(spd, cur) >= 0) {
            cur = adaptive_next(spd, cur);
            const double f0 = info.factor_ms;
            st = timed(&info.factor_ms, [&] { return solver.factor(cur, &hinfo); });
            last_factor_ms = info.factor_ms - f0;
            info.factorizations++;
            info.info = hinfo;
            info.fallback_panels = solver.fallbacks();
            if (st != HDBF_STATUS_SUCCESS || hinfo != 0) break;
            // a classical correction costs two triangular solves against a
            // GMRES step's several: use the new factors that way first.  The
            // first correction is not judged (prev = inf): forward error that
            // the old factors left along the smallest singular directions
            // shows up in the backward error only after it has been spread out
            classical = true;
            prev = INFINITY;
            st = timed(&info.refine_ms, [&] { return solver.correction(buf.R, n, true); });
            continue;
        }
        prev = berr;
        // ---- inner GMRES on M^{-1} A d = M^{-1} r
        int steps = 0;
        st = timed(&info.refine_ms, [&]() -> hdbf_status {
            HDBF_TRY(solver.precond(buf.R, n, buf.V, n, false));
            HDBF_TRY(solver.dots(buf.V, 1, buf.V, sq));
            HDBF_TRY(solver.normalize(buf.V, sq, buf.V));
            HDBF_TRY(to_host(hh.data(), buf.Hd, hbytes));
            std::fill(R.begin(), R.end(), 0.0);
            std::fill(g.begin(), g.end(), 0.0);
            for (int c = 0; c < nrhs; ++c) {
                beta[c] = std::sqrt(hh[(size_t)2 * (m + 1) * nrhs + c]);
                g[(size_t)c * (m + 1)] = beta[c];
            }
            for (int k = 0; k < m; ++k) {
                double* vk = buf.V + (long long)k * vs;
                double* vk1 = buf.V + (long long)(k + 1) * vs;
                HDBF_TRY(solver.matvec(vk, buf.T));
                HDBF_TRY(solver.precond(buf.T, n, vk1, n, false));
                HDBF_TRY(solver.dots(buf.V, k + 1, vk1, h1));
                HDBF_TRY(solver.axpy(buf.V, k + 1, h1, vk1));
                HDBF_TRY(solver.dots(buf.V, k + 1, vk1, h2));
                HDBF_TRY(solver.axpy(buf.V, k + 1, h2, vk1));
                HDBF_TRY(solver.dots(vk1, 1, vk1, sq));
                HDBF_TRY(solver.normalize(vk1, sq, vk1));
                HDBF_TRY(to_host(hh.data(), buf.Hd, hbytes));
                double worst = 0.0;
                for (int c = 0; c < nrhs; ++c) {
                    if (!(beta[c] > 0.0)) continue;
                    double col[64 + 2];
                    for (int i = 0; i <= k; ++i)
                        col[i] = hh[(size_t)i * nrhs + c] + hh[(size_t)(m + 1) * nrhs + (size_t)i * nrhs + c];
                    col[k + 1] = std::sqrt(hh[(size_t)2 * (m + 1) * nrhs + c]);
                    double* csc = cs.data() + (size_t)c * m;
                    double* snc = sn.data() + (size_t)c * m;
                    for (int i = 0; i < k; ++i) {
                        const double t = csc[i] * col[i] + snc[i] * col[i + 1];
                        col[i + 1] = -snc[i] * col[i] + csc[i] * col[i + 1];
                        col[i] = t;
                    }
                    const double den = std::hypot(col[k], col[k + 1]);
                    csc[k] = den > 0.0 ? col[k] / den : 1.0;
                    snc[k] = den > 0.0 ? col[k + 1] / den : 0.0;
                    col[k] = den;
                    double* gc = g.data() + (size_t)c * (m + 1);
                    gc[k + 1] = -snc[k] * gc[k];
                    gc[k] = csc[k] * gc[k];
                    for (int i = 0; i <= k; ++i) R[((size_t)c * (m + 1) + i) * m + k] = col[i];
                    worst = std::max(worst, std::fabs(gc[k + 1]) / beta[c]);
                }
                steps = k + 1;
                if (worst <= inner_tol) break;
            }
            // least squares R y = g per column, then x += V y
            std::fill(y.begin(), y.end(), 0.0);
            for (int c = 0; c < nrhs; ++c) {
                if (!(beta[c] > 0.0)) continue;
                const double* gc = g.data() + (size_t)c * (m + 1);
                for (int i = steps - 1; i >= 0; --i) {
                    double acc = gc[i];
                    for (int j = i + 1; j < steps; ++j)
                        acc -= R[((size_t)c * (m + 1) + i) * m + j] * y[(size_t)j * nrhs + c];
                    const double d = R[((size_t)c * (m + 1) + i) * m + i];
                    y[(size_t)i * nrhs + c] = d != 0.0 ? acc / d : 0.0;
                }
            }
            if (cudaMemcpyAsync(buf.Yd, y.data(), (size_t)steps * nrhs * 8, cudaMemcpyHostToDevice,
                                strm) != cudaSuccess)
                return last_cuda(ctx);
            return solver.combine(buf.V, steps, buf.Yd);
        });
        info.inner_iterations += steps;
        last_step_ms = info.refine_ms - step_start;
    }
    info.final_precision = cur;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (out) *out = info;
    return st;
}

}  // namespace
}  // namespace hdbf

using namespace hdbf;

extern "C" {

hdbf_status hdbf_spotrs(hdbf_handle h, const float* L, int lda, int n, int nrhs, float* B, int ldb)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (n < 0 || nrhs < 0 || (n > 0 && (!L || !B || lda < n || ldb < n)))
        return h->last_status = HDBF_STATUS_INVALID_VALUE;
    return h->last_status = potrs_f32(h, L, lda, n, nrhs, B, ldb);
}

hdbf_status hdbf_sgetrs(hdbf_handle h, const float* LU, int lda, int n, const int* ipiv, int nrhs,
                        float* B, int ldb)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (n < 0 || nrhs < 0 || (n > 0 && (!LU || !B || !ipiv || lda < n || ldb < n)))
        return h->last_status = HDBF_STATUS_INVALID_VALUE;
    if (n == 0 || nrhs == 0) return h->last_status = HDBF_STATUS_SUCCESS;
    hdbf_status st = ensure_ws(h, n);
    if (st != HDBF_STATUS_SUCCESS) return h->last_status = st;
    const size_t need = al((size_t)n * 4) + al((size_t)n * nrhs * 4);
    char* arena = static_cast<char*>(mixed_arena(h, need, &st));
    if (!arena) return h->last_status = st;
    int* perm = reinterpret_cast<int*>(arena);
    float* tmp = reinterpret_cast<float*>(arena + al((size_t)n * 4));
    st = ipiv_to_perm(h, ipiv, n, perm);
    if (st == HDBF_STATUS_SUCCESS) st = gather_rows_perm(h, B, ldb, tmp, n, perm, n, nrhs);
    if (st == HDBF_STATUS_SUCCESS) st = getrs_f32_permuted(h, LU, lda, n, nrhs, tmp, n);
    if (st == HDBF_STATUS_SUCCESS)
        st = cudaMemcpy2DAsync(B, (size_t)ldb * 4, tmp, (size_t)n * 4, (size_t)n * 4, nrhs,
                               cudaMemcpyDeviceToDevice, h->stream) == cudaSuccess
                 ? HDBF_STATUS_SUCCESS
                 : HDBF_STATUS_CUDA_ERROR;
    return h->last_status = st;
}

hdbf_status hdbf_dposv_mixed(hdbf_handle h, hdbf_precision prec, int escalate, const double* A,
                             int lda, int n, int nrhs, const double* B, int ldb, double* X, int ldx,
                             double tol, int max_iter, hdbf_ir_info* out)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = xsv_mixed(h, true, (int)prec, escalate, A, lda, n, nrhs, B, ldb, X,
                                      ldx, tol, max_iter, out);
}

hdbf_status hdbf_dgesv_mixed(hdbf_handle h, hdbf_precision prec, int escalate, const double* A,
                             int lda, int n, int nrhs, const double* B, int ldb, double* X, int ldx,
                             double tol, int max_iter, hdbf_ir_info* out)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = xsv_mixed(h, false, (int)prec, escalate, A, lda, n, nrhs, B, ldb, X,
                                      ldx, tol, max_iter, out);
}

hdbf_status hdbf_dposv_mixed_gmres(hdbf_handle h, hdbf_precision prec, const double* A, int lda,
                                   int n, int nrhs, const double* B, int ldb, double* X, int ldx,
                                   double tol, int max_iter, int max_inner, double inner_tol,
                                   hdbf_ir_info* out)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = gmres_mixed(h, true, prec, A, lda, n, nrhs, B, ldb, X, ldx, tol,
                                        max_iter, max_inner, inner_tol, out);
}

hdbf_status hdbf_dgesv_mixed_gmres(hdbf_handle h, hdbf_precision prec, const double* A, int lda,
                                   int n, int nrhs, const double* B, int ldb, double* X, int ldx,
                                   double tol, int max_iter, int max_inner, double inner_tol,
                                   hdbf_ir_info* out)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = gmres_mixed(h, false, prec, A, lda, n, nrhs, B, ldb, X, ldx, tol,
                                        max_iter, max_inner, inner_tol, out);
}

hdbf_status hdbf_dposv_mixed_auto(hdbf_handle h, hdbf_precision prec, const double* A, int lda,
                                  int n, int nrhs, const double* B, int ldb, double* X, int ldx,
                                  double tol, int max_iter, hdbf_ir_info* out)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = gmres_mixed(h, true, prec, A, lda, n, nrhs, B, ldb, X, ldx, tol,
                                        max_iter, 30, 1e-4, out, true);
}

hdbf_status hdbf_dgesv_mixed_auto(hdbf_handle h, hdbf_precision prec, const double* A, int lda,
                                  int n, int nrhs, const double* B, int ldb, double* X, int ldx,
                                  double tol, int max_iter, hdbf_ir_info* out)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status = gmres_mixed(h, false, prec, A, lda, n, nrhs, B, ldb, X, ldx, tol,
                                        max_iter, 30, 1e-4, out, true);
}

}  // extern "C"
