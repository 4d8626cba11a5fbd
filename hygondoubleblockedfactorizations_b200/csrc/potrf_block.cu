// Cholesky of a diagonal block of order n <= 1024 in ONE cooperative launch,
// optionally with the inverse of its factor.
//
// Replaces the reference's rocsolver_spotrf call on the diagonal block
// (src/potrf/double_blocked_potrf.cpp:34-56, call :334).  The block is cut
// into 64 x 64 tiles (NT = ceil(n / 64) <= 16) and factored right-looking:
// for every tile column k the CTAs solve the tiles below the diagonal against
// the inverse D_k of the factored diagonal tile, then apply the rank-64 update
// to the trailing tiles; with look-ahead, CTA 0 updates tile (k+1, k+1) first
// and factors and inverts it (register-resident potf2) while the other CTAs
// finish the update -- two bounded grid barriers per tile column.  With the
// inverse requested, W = L^{-1} (lower, the strictly upper tiles zeroed) is
// formed by recursive doubling over tile blocks: for siblings A and C,
// W(C,A) = -W(C,C) (L(C,A) W(A,A)), two GEMM phases per level.
// A recursive factorization of the same block issues ~100 small launches.
//
// Pivot test and info follow LAPACK xPOTRF: the first column whose updated
// diagonal is not > 0 (or is NaN) stops the factorization and info =
// info_base + column + 1 (first failure wins); a block whose info is already
// non-zero is left untouched.  Every grid-barrier wait is bounded: on expiry
// the kernel records a timeout, and later barriers return at once.
#include <algorithm>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int kT = 64;        // tile
constexpr int kThreads = 256;
constexpr int kMaxNT = 16;    // n <= 1024
constexpr int kLdS = 68;      // padded shared row (float4-aligned)

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

struct Sync {
    unsigned* ctr;
    int* fail;
    int* abort_flag;
    int* err;
    unsigned G;
    unsigned count;  // barriers passed by this CTA
    unsigned limit;  // poll limit (the handle's, spin_limit_of)
};

// Grid barrier: arrive (counter += 1 per CTA), wait until all G CTAs of this
// round arrived.  Bounded; once any CTA gave up, later waits return at once.
__device__ void grid_barrier(Sync& s)
{
    __syncthreads();
    s.count += 1;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(s.ctr, 1u);
        const unsigned target = s.count * s.G;
        unsigned polls = 0;
        while (ld_acquire_u32(s.ctr) < target) {
            if (*reinterpret_cast<volatile int*>(s.abort_flag)) break;
            if (++polls > s.limit) {
                atomicCAS(s.err, 0, kErrTimeout);
                atomicExch(s.abort_flag, 1);
                break;
            }
            if (polls > 64) __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

// Two 64 x 64 tiles into shared memory, every global load of the thread in
// flight before the first shared store (the tiles live in L2, so the loads'
// latency, not their bandwidth, sets the cost).  Tile X (X = A, B) is the
// column-major block src (leading dimension ld, entries outside rows x cols
// read as zero); TX = false stores it k-major, dst[k][m] = src(m, k), and
// TX = true transposed, dst[k][n] = src(k, n), both with row pitch kLdS.
struct TileSrc {
    const float* src;
    long long ld;
    int rows, cols;
};
template <bool TA, bool TB>
__device__ __forceinline__ void load_pair(float* dA, TileSrc a, float* dB, TileSrc b)
{
    constexpr int kPer = kT * kT / kThreads;  // 16 elements per thread and tile
    float va[kPer], vb[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int q = threadIdx.x + u * kThreads, c = q >> 6, r = q & 63;
        va[u] = (r < a.rows && c < a.cols) ? __ldcg(a.src + (long long)c * a.ld + r) : 0.f;
        vb[u] = (r < b.rows && c < b.cols) ? __ldcg(b.src + (long long)c * b.ld + r) : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int q = threadIdx.x + u * kThreads, c = q >> 6, r = q & 63;
        dA[TA ? r * kLdS + c : c * kLdS + r] = va[u];
        dB[TB ? r * kLdS + c : c * kLdS + r] = vb[u];
    }
}

// acc[i][j] += sum_k As[k][ty*4+i] * Bs[k][tx*4+j]
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

// Register-resident Cholesky of the nb x nb (nb <= 64) lower tile at T
// (thread (r, g) holds T(r, g + 4i), i < 16).  Returns the first failing
// column or -1 (uniform over the CTA).
__device__ int potf2_tile(float* T, long long ld, int nb, float* lcol, float* s_d)
{
    const int tid = threadIdx.x, r = tid & 63, g = tid >> 6;
    float a[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int c = g + 4 * i;
        a[i] = (r < nb && c < nb && r >= c) ? __ldcg(T + (long long)c * ld + r) : 0.f;
    }
    int failed_at = -1;
    for (int j = 0; j < nb; ++j) {
        const int gj = j & 3, ij = j >> 2;
        float own = 0.f;
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (i == ij) own = a[i];
        if (g == gj && r == j) *s_d = own;
        __syncthreads();
        const float d = *s_d;
        if (!(d > 0.f)) {
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
        if (r < nb && c < nb && r >= c) T[(long long)c * ld + r] = a[i];
    }
    return failed_at;
}

// D = L^{-1} for the nb x nb lower tile L (padded with the identity to 64):
// thread t < 64 solves L x = e_t by forward substitution over a shared copy.
// D is written column-major with leading dimension 64 (D[c * 64 + r]).
__device__ void tri_inv_tile(const float* L, long long ld, int nb, float* Ls /*64 x 65*/,
                             float* D)
{
    {
        float v[kT * kT / kThreads];  // all loads in flight before the first store
#pragma unroll
        for (int u = 0; u < kT * kT / kThreads; ++u) {
            const int q = threadIdx.x + u * kThreads, c = q >> 6, r = q & 63;
            v[u] = (r < nb && c < nb && r >= c) ? __ldcg(L + (long long)c * ld + r) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kT * kT / kThreads; ++u) {
            const int q = threadIdx.x + u * kThreads, c = q >> 6, r = q & 63;
            Ls[r * 65 + c] = v[u];
        }
    }
    __syncthreads();
    const int t = threadIdx.x;
    if (t < kT) {
        float x[kT];
#pragma unroll
        for (int i = 0; i < kT; ++i) x[i] = (i == t) ? 1.f : 0.f;
#pragma unroll
        for (int k = 0; k < kT; ++k) {
            if (k < nb) {
                x[k] = x[k] / Ls[k * 65 + k];
#pragma unroll
                for (int i = k + 1; i < kT; ++i) x[i] = fmaf(-Ls[i * 65 + k], x[k], x[i]);
            }
        }
#pragma unroll
        for (int i = 0; i < kT; ++i) D[t * kT + i] = x[i];  // column t
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads, 1)
potrf_block_kernel(int n, float* A, long long lda, int* info, int info_base, float* W,
                   long long ldw, float* dinv, float* Tsc, unsigned* ctr, int* fail,
                   int* abort_flag, int* err, const int* run_if)
{
    __shared__ __align__(16) float As[kT * kLdS];
    __shared__ __align__(16) float Bs[kT * kLdS];
    __shared__ float lcol[kT];
    __shared__ float s_d;
    __shared__ int s_flag;
    const int NT = (n + kT - 1) / kT;
    const int cta = blockIdx.x;
    const unsigned G = gridDim.x;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    Sync sy{ctr, fail, abort_flag, err, G, 0u, spin_limit_of(err)};
    auto tile = [&](int i, int j) { return A + (long long)(j * kT) * lda + i * kT; };
    auto ext = [&](int i) { return min(kT, n - i * kT); };

    if (tid == 0)
        s_flag = ((info && *reinterpret_cast<volatile int*>(info) != 0) ||
                  (run_if && *reinterpret_cast<const volatile int*>(run_if) == 0))
                     ? 1
                     : 0;
    __syncthreads();
    const bool skip = s_flag != 0;  // same value in every CTA: read before any write
    grid_barrier(sy);
    if (skip) return;

    // Factor (and invert) diagonal tile k on this CTA; false on a bad pivot.
    auto factor_diag = [&](int k) -> bool {
        const int f = potf2_tile(tile(k, k), lda, ext(k), lcol, &s_d);
        if (f >= 0) {
            if (tid == 0) {
                if (info) atomicCAS(info, 0, info_base + k * kT + f + 1);
                atomicExch(fail, 1);
            }
            return false;
        }
        __syncthreads();
        tri_inv_tile(tile(k, k), lda, ext(k), As, dinv + (long long)k * kT * kT);
        return true;
    };
    // A(i,j) -= L(i,k) L(j,k)^T (lower part only on the diagonal)
    auto update_tile = [&](int k, int i, int j) {
        load_pair<false, false>(As, {tile(i, k), lda, ext(i), ext(k)}, Bs,
                                {tile(j, k), lda, ext(j), ext(k)});
        __syncthreads();
        float acc[4][4] = {};
        tile_mma(acc, As, Bs);
        float* T = tile(i, j);
        float old[4][4];  // all loads in flight before the first store
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = ty * 4 + a, c = tx * 4 + b;
                old[a][b] = (r < ext(i) && c < ext(j) && (i != j || r >= c))
                                ? __ldcg(T + (long long)c * lda + r)
                                : 0.f;
            }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = ty * 4 + a, c = tx * 4 + b;
                if (r < ext(i) && c < ext(j) && (i != j || r >= c))
                    T[(long long)c * lda + r] = old[a][b] - acc[a][b];
            }
        __syncthreads();
    };
    auto failed = [&]() -> bool {
        if (tid == 0) s_flag = *reinterpret_cast<volatile int*>(fail) |
                               *reinterpret_cast<volatile int*>(abort_flag);
        __syncthreads();
        return s_flag != 0;
    };

    // Right-looking over tile columns with look-ahead: during the trailing
    // update of step k, CTA 0 first updates tile (k+1, k+1) and factors it
    // while the other CTAs update the remaining tiles.
    if (cta == 0) factor_diag(0);
    grid_barrier(sy);
    bool ok = !failed();
    for (int k = 0; k < NT - 1 && ok; ++k) {
        // P2: L(i,k) = A(i,k) D_k^T for i > k
        for (int i = k + 1 + cta; i < NT; i += G) {
            load_pair<false, false>(As, {tile(i, k), lda, ext(i), ext(k)}, Bs,
                                    {dinv + (long long)k * kT * kT, kT, ext(k), ext(k)});
            __syncthreads();
            float acc[4][4] = {};
            tile_mma(acc, As, Bs);
            float* T = tile(i, k);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const int r = ty * 4 + a, c = tx * 4 + b;
                    if (r < ext(i) && c < ext(k)) T[(long long)c * lda + r] = acc[a][b];
                }
            __syncthreads();
        }
        grid_barrier(sy);
        // P3 (+ P1 of step k+1 on CTA 0): pairs t >= 1 on CTAs 1.., t = 0 is
        // tile (k+1, k+1)
        const int rem = NT - 1 - k;
        const int pairs = rem * (rem + 1) / 2;
        if (cta == 0) {
            update_tile(k, k + 1, k + 1);
            factor_diag(k + 1);
        }
        const int workers = G > 1 ? (int)G - 1 : 1;
        const int first = G > 1 ? cta - 1 : 0;
        if (G == 1 || cta > 0) {
            for (int t = 1 + first; t < pairs; t += workers) {
                int i = k + 1, left = t;
                while (left > i - (k + 1)) { left -= i - k; ++i; }
                update_tile(k, i, k + 1 + left);
            }
        }
        grid_barrier(sy);
        if (failed()) { ok = false; break; }
    }
    if (!ok || !W) return;

    // W = L^{-1} by recursive doubling over tile blocks: for sibling blocks
    // A = [b, b+s) and C = [b+s, b+2s) (tiles), W(C,A) = -W(C,C) (L(C,A) W(A,A)),
    // T = L(C,A) W(A,A) kept in scratch at the W(C,A) position.
    // Setup: diagonal tiles D_i, strictly upper tiles zero.
    for (int t = cta; t < NT * NT; t += G) {
        const int i = t % NT, j = t / NT;
        if (i < j) {
            for (int q = tid; q < kT * kT; q += kThreads) {
                const int c = q >> 6, r = q & 63;
                if (r < ext(i) && c < ext(j)) W[(long long)(j * kT + c) * ldw + i * kT + r] = 0.f;
            }
        } else if (i == j) {
            const float* D = dinv + (long long)i * kT * kT;
            for (int q = tid; q < kT * kT; q += kThreads) {
                const int c = q >> 6, r = q & 63;
                if (r < ext(i) && c < ext(i))
                    W[(long long)(i * kT + c) * ldw + i * kT + r] = __ldcg(D + c * kT + r);
            }
        }
    }
    grid_barrier(sy);
    auto wt = [&](int i, int j) { return W + (long long)(j * kT) * ldw + i * kT; };
    auto tt = [&](int i, int j) { return Tsc + (long long)(j * kT) * ldw + i * kT; };
    for (int st = 1; st < NT; st *= 2) {
        // tiles (ci, aj) of every pair: C rows [b+st, min(b+2st, NT)), A cols [b, b+st)
        const int npair = (NT + 2 * st - 1) / (2 * st);
        const int per = st * st;
        // phase A: T(ci, aj) = sum_{m=aj}^{b+st-1} L(ci, m) W(m, aj)
        for (int t = cta; t < npair * per; t += G) {
            const int pr = t / per, q = t - pr * per;
            const int b = pr * 2 * st;
            const int ci = b + st + q / st, aj = b + q % st;
            if (ci >= NT) continue;
            float acc[4][4] = {};
            for (int m = aj; m < b + st; ++m) {
                load_pair<false, true>(As, {tile(ci, m), lda, ext(ci), ext(m)}, Bs,
                                       {wt(m, aj), ldw, ext(m), ext(aj)});
                __syncthreads();
                tile_mma(acc, As, Bs);
                __syncthreads();
            }
            float* T = tt(ci, aj);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    const int r = ty * 4 + a, c = tx * 4 + bb;
                    if (r < ext(ci) && c < ext(aj)) T[(long long)c * ldw + r] = acc[a][bb];
                }
        }
        grid_barrier(sy);
        // phase B: W(ci, aj) = -sum_{m=b+st}^{ci} W(ci, m) T(m, aj)
        for (int t = cta; t < npair * per; t += G) {
            const int pr = t / per, q = t - pr * per;
            const int b = pr * 2 * st;
            const int ci = b + st + q / st, aj = b + q % st;
            if (ci >= NT) continue;
            float acc[4][4] = {};
            for (int m = b + st; m <= ci; ++m) {
                load_pair<false, true>(As, {wt(ci, m), ldw, ext(ci), ext(m)}, Bs,
                                       {tt(m, aj), ldw, ext(m), ext(aj)});
                __syncthreads();
                tile_mma(acc, As, Bs);
                __syncthreads();
            }
            float* Wp = wt(ci, aj);
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    const int r = ty * 4 + a, c = tx * 4 + bb;
                    if (r < ext(ci) && c < ext(aj)) Wp[(long long)c * ldw + r] = -acc[a][bb];
                }
        }
        grid_barrier(sy);
    }
}

}  // namespace

int potrf_block_max_n() { return kT * kMaxNT; }

hdbf_status potrf_block(hdbf_context* ctx, int n, float* A, long long lda, int* info,
                        int info_base, float* W, long long ldw)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    if (n > kT * kMaxNT || lda < n || (W && ldw < n)) return HDBF_STATUS_INVALID_VALUE;
    // ws_skinny holds 256 * ws_n floats: >= n * ldw once ws_n >= max(n, ldw * n / 256)
    const long long need = W ? ((long long)ldw * n + 255) / 256 : 0;
    HDBF_TRY(ensure_ws(ctx, (int)std::max<long long>(n, std::max<long long>(need, 64))));
    const int NT = (n + kT - 1) / kT;
    int G = NT * (NT - 1) / 2;
    if (W && NT * NT > G) G = NT * NT;  // the W set-up pass touches NT^2 tiles
    if (G > ctx->sm_count) G = ctx->sm_count;
    if (G < 1) G = 1;
    int* sm = ctx->dev_small + kSmallBlockBar;
    if (cudaMemsetAsync(sm, 0, 3 * sizeof(int), ctx->stream) != cudaSuccess) return last_cuda(ctx);
    unsigned* ctr = reinterpret_cast<unsigned*>(sm);
    int* fail = sm + 1;
    int* abort_flag = sm + 2;
    int* err = ctx->dev_small + kSmallErr;
    float* dinv = ws_inv(ctx);
    float* Tsc = ws_skinny(ctx);  // n x n scratch (leading dimension ldw) for the inverse
    const double flops = (double)n * n * n / 3.0 + (W ? (double)n * n * n / 3.0 : 0.0);
    ProfScope prof(ctx, kClsPotrfBlock, flops, 8.0 * n * n, n, n, n);
    const int* run_if = ctx->run_if;
    void* args[] = {&n, &A, &lda, &info, &info_base, &W, &ldw, &dinv, &Tsc, &ctr, &fail,
                    &abort_flag, &err, &run_if};
    const cudaError_t e = cudaLaunchCooperativeKernel((const void*)potrf_block_kernel, dim3(G),
                                                      dim3(kThreads), args, 0, ctx->stream);
    ctx->launches++;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    return HDBF_STATUS_SUCCESS;
}

}  // namespace hdbf
