// Batched uneven factor-and-solve in one persistent launch.
//
// Thousands of independent small systems (Cholesky: n <= 512, LU with partial
// pivoting: n <= 768, one right-hand side each) are processed by a grid of
// persistent CTAs that pull matrix indices from a device work queue (largest
// work first, so the tail is short).  Each CTA factors its matrix in place with
// a right-looking blocked algorithm (panel width 32) whose panel, triangular
// inverse and trailing-update operands live in shared memory, then solves its
// right-hand side in place.  No reference counterpart (the reference factors
// one matrix per call); the per-matrix arithmetic follows LAPACK's blocked
// xPOTRF / xGETRF (first maximum pivot, reciprocal scaling, info = first
// failing column).
#include <algorithm>
#include <cfloat>
#include <climits>
#include <vector>

#include "internal.h"
#include "hdbf/batched.h"

namespace hdbf {
namespace {

constexpr int PW = 32;         // panel width
constexpr int kMaxChol = 512;  // largest Cholesky order
constexpr int kMaxLu = 768;    // largest LU order

struct BatchArgs {
    int count;
    const int* order;  // processing order (indices into the arrays below)
    const int* op;     // 0 = POTRF + POTRS, 1 = GETRF + GETRS
    const int* n;
    const int* lda;
    float* const* A;
    float* const* b;
    int* const* ipiv;
    int* info;
    unsigned* queue;
};

template <int T>
__device__ __forceinline__ void block_argmax(float v, int i, float* rv, int* ri, float* out_v,
                                             int* out_i)
{
    // largest v, lowest index on ties; i == INT_MAX marks "no candidate"
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_down_sync(0xffffffffu, v, off);
        const int oi = __shfl_down_sync(0xffffffffu, i, off);
        if (oi != INT_MAX && (i == INT_MAX || ov > v || (ov == v && oi < i))) { v = ov; i = oi; }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { rv[warp] = v; ri[warp] = i; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < T / 32; ++w)
            if (ri[w] != INT_MAX && (i == INT_MAX || rv[w] > v || (rv[w] == v && ri[w] < i))) {
                v = rv[w];
                i = ri[w];
            }
        *out_v = v;
        *out_i = i;
    }
    __syncthreads();
}

// ------------------------------------------------------------------ Cholesky
template <int T>
__device__ void chol_solve(float* A, int n, long long lda, float* b, int* info, float* sm)
{
    float* S = sm;                     // 32 x 33 diagonal block (col-major, ld 33)
    float* Inv = S + PW * 33;          // 32 x 33 inverse of the diagonal block
    float* P = Inv + PW * 33;          // panel below the diagonal block: m x 32, ld kMaxChol
    float* red_v = P + kMaxChol * PW;  // reductions
    __shared__ int s_fail;
    const int tid = threadIdx.x;
    if (tid == 0) s_fail = 0;
    __syncthreads();
    for (int k = 0; k < n; k += PW) {
        const int kb = min(PW, n - k);
        const int m = n - k - kb;
        for (int idx = tid; idx < PW * PW; idx += T) {
            const int c = idx / PW, r = idx % PW;
            S[c * 33 + r] = (r < kb && c < kb && r >= c) ? A[(long long)(k + c) * lda + k + r] : 0.f;
        }
        __syncthreads();
        // unblocked Cholesky of the diagonal block
        for (int j = 0; j < kb; ++j) {
            const float d = S[j * 33 + j];
            __syncthreads();
            if (!(d > 0.f)) {
                if (tid == 0) {
                    s_fail = k + j + 1;
                    A[(long long)(k + j) * lda + k + j] = d;
                }
                break;
            }
            const float sd = sqrtf(d), rcp = 1.0f / sd;
            if (tid == 0) S[j * 33 + j] = sd;
            for (int i = j + 1 + tid; i < kb; i += T) S[j * 33 + i] *= rcp;
            __syncthreads();
            for (int idx = tid; idx < kb * kb; idx += T) {
                const int c = idx / kb, r = idx % kb;
                if (c > j && r >= c) S[c * 33 + r] -= S[j * 33 + r] * S[j * 33 + c];
            }
            __syncthreads();
        }
        __syncthreads();
        if (s_fail) break;
        for (int idx = tid; idx < kb * kb; idx += T) {
            const int c = idx / kb, r = idx % kb;
            if (r >= c) A[(long long)(k + c) * lda + k + r] = S[c * 33 + r];
        }
        // inverse of the diagonal block (thread t < kb: column t)
        if (tid < PW) {
            float x[PW];
#pragma unroll
            for (int i = 0; i < PW; ++i) x[i] = (i == tid) ? 1.f : 0.f;
#pragma unroll
            for (int q = 0; q < PW; ++q) {
                if (q < kb) {
                    x[q] = x[q] / S[q * 33 + q];
#pragma unroll
                    for (int i = q + 1; i < PW; ++i)
                        if (i < kb) x[i] = fmaf(-S[q * 33 + i], x[q], x[i]);
                }
            }
#pragma unroll
            for (int i = 0; i < PW; ++i) Inv[tid * 33 + i] = x[i];
        }
        __syncthreads();
        // panel: P(r, :) = A21(r, :) * Inv^T, rows k+kb .. n
        for (int r = tid; r < m; r += T) {
            float row[PW];
#pragma unroll
            for (int c = 0; c < PW; ++c) row[c] = c < kb ? A[(long long)(k + c) * lda + k + kb + r] : 0.f;
#pragma unroll
            for (int c = 0; c < PW; ++c) {
                float s = 0.f;
#pragma unroll
                for (int q = 0; q < PW; ++q)
                    if (q <= c) s = fmaf(row[q], Inv[q * 33 + c], s);
                if (c < kb) {
                    P[c * kMaxChol + r] = s;
                    A[(long long)(k + c) * lda + k + kb + r] = s;
                }
            }
        }
        __syncthreads();
        // trailing lower update A22 -= P P^T on 64 x (T/4) tiles
        constexpr int TC = T / 16;  // tile columns: 16 row-groups of 4 x (T/16) col-groups of 4
        for (int j0 = 0; j0 < m; j0 += TC * 4) {
            for (int i0 = j0; i0 < m; i0 += 64) {
                const int rr = i0 + (tid % 16) * 4, cc = j0 + (tid / 16) * 4;
                float acc[4][4] = {};
                for (int q = 0; q < kb; ++q) {
                    float a[4], bq[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        a[u] = (rr + u < m) ? P[q * kMaxChol + rr + u] : 0.f;
                        bq[u] = (cc + u < m) ? P[q * kMaxChol + cc + u] : 0.f;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], bq[v], acc[u][v]);
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int c = cc + v;
                    if (c >= m) continue;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int r = rr + u;
                        if (r < m && r >= c)
                            A[(long long)(k + kb + c) * lda + k + kb + r] -= acc[u][v];
                    }
                }
            }
        }
        __syncthreads();
    }
    (void)red_v;
    if (s_fail) {
        if (tid == 0) *info = s_fail;
        return;
    }
    if (tid == 0) *info = 0;
    // Solve L y = b then L^T x = y (b in shared memory, one column).
    float* x = P;  // reuse
    for (int i = tid; i < n; i += T) x[i] = b[i];
    __syncthreads();
    for (int j = 0; j < n; ++j) {  // forward, column-oriented
        if (tid == 0) x[j] = x[j] / A[(long long)j * lda + j];
        __syncthreads();
        const float xj = x[j];
        for (int i = j + 1 + tid; i < n; i += T) x[i] = fmaf(-A[(long long)j * lda + i], xj, x[i]);
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; --j) {  // backward with L^T: x_j = (y_j - sum_{i>j} L_ij x_i) / L_jj
        float s = 0.f;
        for (int i = j + 1 + tid; i < n; i += T) s = fmaf(A[(long long)j * lda + i], x[i], s);
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if ((tid & 31) == 0) red_v[tid >> 5] = s;
        __syncthreads();
        if (tid == 0) {
            float t = 0.f;
            for (int w = 0; w < T / 32; ++w) t += red_v[w];
            x[j] = (x[j] - t) / A[(long long)j * lda + j];
        }
        __syncthreads();
    }
    for (int i = tid; i < n; i += T) b[i] = x[i];
}

// ------------------------------------------------------------------ LU
template <int T>
__device__ void lu_solve(float* A, int n, long long lda, float* b, int* ipiv, int* info, float* sm)
{
    float* L11 = sm;                  // 32 x 33 unit lower block
    float* L21 = L11 + PW * 33;       // m x 32, ld kMaxLu
    float* U12 = L21 + kMaxLu * PW;   // 32 x m, row-major ld kMaxLu
    float* red_v = U12 + PW * kMaxLu;
    __shared__ int red_i[T / 32];
    __shared__ float s_pv;
    __shared__ int s_pi, s_info;
    const int tid = threadIdx.x;
    if (tid == 0) s_info = 0;
    __syncthreads();
    for (int k = 0; k < n; k += PW) {
        const int kb = min(PW, n - k);
        const int m = n - k - kb;
        for (int j = k; j < k + kb; ++j) {
            float v = -1.f;
            int vi = INT_MAX;
            for (int i = j + tid; i < n; i += T) {
                const float a = fabsf(A[(long long)j * lda + i]);
                if (vi == INT_MAX || a > v) { v = a; vi = i; }
            }
            block_argmax<T>(v, vi, red_v, red_i, &s_pv, &s_pi);
            const int p = s_pi;
            if (tid == 0) ipiv[j] = p + 1;
            const float piv = A[(long long)j * lda + p];
            __syncthreads();  // every thread has read the pivot before the swap rewrites it
            if (p != j)  // swap entire rows j and p
                for (int c = tid; c < n; c += T) {
                    float* cj = A + (long long)c * lda;
                    const float t = cj[j];
                    cj[j] = cj[p];
                    cj[p] = t;
                }
            __syncthreads();
            if (piv != 0.f) {
                const bool recip = fabsf(piv) >= FLT_MIN;
                const float rcp = 1.0f / piv;
                for (int i = j + 1 + tid; i < n; i += T) {
                    float* a = A + (long long)j * lda + i;
                    *a = recip ? *a * rcp : *a / piv;
                }
            } else if (tid == 0 && s_info == 0) {
                s_info = j + 1;
            }
            __syncthreads();
            // rank-1 update of the panel columns j+1 .. k+kb
            const int pc = k + kb - j - 1;
            const int pr = n - j - 1;
            for (int idx = tid; idx < pc * pr; idx += T) {
                const int c = j + 1 + idx / pr, r = j + 1 + idx % pr;
                A[(long long)c * lda + r] = fmaf(-A[(long long)j * lda + r], A[(long long)c * lda + j],
                                                 A[(long long)c * lda + r]);
            }
            __syncthreads();
        }
        if (m <= 0) break;
        // L11 and L21 into shared memory
        for (int idx = tid; idx < PW * PW; idx += T) {
            const int c = idx / PW, r = idx % PW;
            L11[c * 33 + r] = (r > c && r < kb && c < kb) ? A[(long long)(k + c) * lda + k + r] : 0.f;
        }
        for (int idx = tid; idx < m * kb; idx += T) {
            const int c = idx / m, r = idx % m;
            L21[c * kMaxLu + r] = A[(long long)(k + c) * lda + k + kb + r];
        }
        __syncthreads();
        // U12 = L11^{-1} A12 (thread per column)
        for (int c = tid; c < m; c += T) {
            float x[PW];
            float* col = A + (long long)(k + kb + c) * lda + k;
#pragma unroll
            for (int r = 0; r < PW; ++r) x[r] = r < kb ? col[r] : 0.f;
#pragma unroll
            for (int q = 0; q < PW; ++q)
#pragma unroll
                for (int r = q + 1; r < PW; ++r) x[r] = fmaf(-L11[q * 33 + r], x[q], x[r]);
#pragma unroll
            for (int r = 0; r < PW; ++r)
                if (r < kb) {
                    col[r] = x[r];
                    U12[r * kMaxLu + c] = x[r];
                }
        }
        __syncthreads();
        // A22 -= L21 U12
        constexpr int TC = T / 16;
        for (int j0 = 0; j0 < m; j0 += TC * 4) {
            for (int i0 = 0; i0 < m; i0 += 64) {
                const int rr = i0 + (tid % 16) * 4, cc = j0 + (tid / 16) * 4;
                float acc[4][4] = {};
                for (int q = 0; q < kb; ++q) {
                    float a[4], bq[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        a[u] = (rr + u < m) ? L21[q * kMaxLu + rr + u] : 0.f;
                        bq[u] = (cc + u < m) ? U12[q * kMaxLu + cc + u] : 0.f;
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], bq[v], acc[u][v]);
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const int c = cc + v;
                    if (c >= m) continue;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int r = rr + u;
                        if (r < m) A[(long long)(k + kb + c) * lda + k + kb + r] -= acc[u][v];
                    }
                }
            }
        }
        __syncthreads();
    }
    if (tid == 0) *info = s_info;
    if (s_info) return;
    // Solve: x = U^{-1} L^{-1} P b
    float* x = L21;
    for (int i = tid; i < n; i += T) x[i] = b[i];
    __syncthreads();
    if (tid == 0)
        for (int i = 0; i < n; ++i) {
            const int p = ipiv[i] - 1;
            if (p != i) {
                const float t = x[i];
                x[i] = x[p];
                x[p] = t;
            }
        }
    __syncthreads();
    for (int j = 0; j < n; ++j) {  // unit lower, column-oriented
        const float xj = x[j];
        for (int i = j + 1 + tid; i < n; i += T) x[i] = fmaf(-A[(long long)j * lda + i], xj, x[i]);
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; --j) {  // upper, column-oriented
        if (tid == 0) x[j] = x[j] / A[(long long)j * lda + j];
        __syncthreads();
        const float xj = x[j];
        for (int i = tid; i < j; i += T) x[i] = fmaf(-A[(long long)j * lda + i], xj, x[i]);
        __syncthreads();
    }
    for (int i = tid; i < n; i += T) b[i] = x[i];
}

template <int T>
__global__ void __launch_bounds__(T) batched_factor_solve_kernel(BatchArgs a)
{
    extern __shared__ float sm[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(a.queue, 1u);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= a.count) break;
        const int idx = a.order[it];
        const int n = a.n[idx];
        if (n <= 0) continue;
        if (a.op[idx] == 0) {
            if (n <= kMaxChol) chol_solve<T>(a.A[idx], n, a.lda[idx], a.b[idx], a.info + idx, sm);
        } else {
            if (n <= kMaxLu) lu_solve<T>(a.A[idx], n, a.lda[idx], a.b[idx], a.ipiv[idx], a.info + idx, sm);
        }
        __syncthreads();
    }
}

constexpr size_t kSmemFloats =
    (size_t)PW * 33 + (size_t)kMaxLu * PW + (size_t)PW * kMaxLu + 64;  // LU layout is the larger

template <int T>
hdbf_status launch_batched(hdbf_context* ctx, const BatchArgs& a, int ctas)
{
    const size_t smem = kSmemFloats * sizeof(float);
    batched_factor_solve_kernel<T><<<ctas, T, smem, ctx->stream>>>(a);
    ctx->launches++;
    return last_cuda(ctx);
}

}  // namespace

void configure_batched_kernels(hdbf_context* ctx)
{
    (void)ctx;
    const int smem = (int)(kSmemFloats * sizeof(float));
    cudaFuncSetAttribute(batched_factor_solve_kernel<128>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(batched_factor_solve_kernel<256>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(batched_factor_solve_kernel<512>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaGetLastError();
}

}  // namespace hdbf

using namespace hdbf;

extern "C" {

int hdbf_batched_num_variants(void) { return 3; }

hdbf_status hdbf_batched_factor_solve(hdbf_handle h, int variant, int count, const int* order,
                                      const int* op, const int* n, const int* lda, float* const* A,
                                      float* const* b, int* const* ipiv, int* info,
                                      unsigned int* queue)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (count < 0 || variant < 0 || variant > 2) return h->last_status = HDBF_STATUS_INVALID_VALUE;
    if (count == 0) return h->last_status = HDBF_STATUS_SUCCESS;
    if (!order || !op || !n || !lda || !A || !b || !ipiv || !info || !queue)
        return h->last_status = HDBF_STATUS_INVALID_VALUE;
    BatchArgs a{count, order, op, n, lda, A, b, ipiv, info, queue};
    const std::vector<long long> key = {40, variant, count, (long long)order, (long long)op,
                                        (long long)n, (long long)lda, (long long)A, (long long)b,
                                        (long long)ipiv, (long long)info, (long long)queue};
    const int ctas = h->sm_count;  // one persistent CTA per SM (shared memory bound)
    return h->last_status = run_graph(h, key, [&]() -> hdbf_status {
        cudaMemsetAsync(queue, 0, sizeof(unsigned int), h->stream);
        ProfScope prof(h, kClsBatched, 0.0, 0.0);
        if (variant == 0) return launch_batched<128>(h, a, ctas);
        if (variant == 1) return launch_batched<256>(h, a, ctas);
        return launch_batched<512>(h, a, ctas);
    });
}

}  // extern "C"
