// Batched uneven factor-and-solve in one persistent launch.
//
// Thousands of independent small systems (Cholesky: n <= 512, LU with partial
// pivoting: n <= 768, one right-hand side each) are processed by a grid of
// persistent CTAs (several per SM) that pull matrix indices from a device
// work queue (largest work first, so the tail is short).  Each CTA factors its
// matrix in place, right-looking with panels of PW columns:
//   * the panel (all rows below the diagonal, PW columns) is copied into
//     shared memory and factored there with two barriers per column -- the
//     pivot search of column j+1 is fused into the rank-1 update of column j;
//   * LU: the panel's row interchanges are composed into at most 2 PW row
//     moves and applied to the other columns with one gather / scatter per
//     column (every load of a column before its first store);
//   * the trailing update runs over 64-column chunks: the chunk's U12 block
//     (LU: a unit-lower triangular solve against the panel's diagonal block,
//     one thread per column) and then A22 -= L21 U12 (Cholesky: L21 L21^T,
//     lower part only) with 8 x 4 register tiles fed by 128-bit shared loads;
// then solves its right-hand side with blocked substitutions (one warp per
// diagonal block, all threads on the off-diagonal block rows).
// The launch shape is a variant: threads per CTA and panel width; the
// shared-memory footprint of the panel width sets the CTAs per SM.
// No reference counterpart (the reference factors one matrix per call); the
// per-matrix arithmetic follows LAPACK's xPOTRF / xGETRF (first maximum
// pivot, reciprocal scaling unless |pivot| < FLT_MIN, info = first failing
// column; LU keeps factoring after a zero pivot, Cholesky stops).
#include <algorithm>
#include <cfloat>
#include <climits>
#include <vector>

#include "internal.h"
#include "hdbf/batched.h"

namespace hdbf {
namespace {

constexpr int kMaxChol = 512;  // largest Cholesky order
constexpr int kMaxLu = 768;    // largest LU order
constexpr int kLdp = kMaxLu + 8;  // panel rows (padding for 8-row register tiles)
constexpr int kChunk = 64;        // trailing-update columns per pass
constexpr int kUbLd = kChunk + 4;

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

// Shared-memory footprint (floats) for panel width PW.
template <int PW>
constexpr size_t smem_floats()
{
    return (size_t)kLdp * PW          // panel
           + (size_t)PW * kUbLd       // U12 chunk
           + (size_t)kMaxLu           // row map (factor) / solution (solve)
           + (size_t)2 * PW * 2       // move list
           + 2 * PW + 64;             // column scratch, reductions
}

template <int T, int PW>
struct Smem {
    float* P;      // panel P[c * kLdp + r], r relative to the panel's first row
    float* Ub;     // U12 chunk Ub[q * kUbLd + c]
    int* rowmap;   // LU: composed swaps of the panel (aliases x)
    float* x;      // solve vector
    int* mv;       // moves: mv[i] = source row, mv[2 PW + i] = target row
    float* col;    // scaled column entries / dot products (2 PW)
    float* rv;     // reductions (T / 32)
    int* ri;
    __device__ explicit Smem(float* sm)
    {
        P = sm;
        Ub = P + (size_t)kLdp * PW;
        x = Ub + (size_t)PW * kUbLd;
        rowmap = reinterpret_cast<int*>(x);
        mv = reinterpret_cast<int*>(x + kMaxLu);
        col = reinterpret_cast<float*>(mv + 4 * PW);
        rv = col + 2 * PW;
        ri = reinterpret_cast<int*>(rv + 32);
    }
};

// (v, i) beats (bv, bi): a real row beats none, then larger |a|, then the
// lower row (LAPACK ISAMAX returns the first maximum).
__device__ __forceinline__ bool better(float v, int i, float bv, int bi)
{
    if (i == INT_MAX) return false;
    if (bi == INT_MAX) return true;
    return v > bv || (v == bv && i < bi);
}

// Block-wide argmax of the per-thread candidates; every thread gets the row.
template <int T>
__device__ __forceinline__ int block_argmax(float v, int i, float* rv, int* ri)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i, off);
        if (better(ov, oi, v, i)) { v = ov; i = oi; }
    }
    if ((threadIdx.x & 31) == 0) { rv[threadIdx.x >> 5] = v; ri[threadIdx.x >> 5] = i; }
    __syncthreads();
    v = rv[0];
    i = ri[0];
#pragma unroll
    for (int w = 1; w < T / 32; ++w)
        if (better(rv[w], ri[w], v, i)) { v = rv[w]; i = ri[w]; }
    return i;
}

// ------------------------------------------------------------ panel kernels
// Pivoted LU of the m x kb panel P (m rows from the diagonal down).  piv[j]
// receives the panel row swapped with row j.  Returns the first zero-pivot
// column + 1 (0: none); the factorization continues past it, as xGETF2.
template <int T, int PW>
__device__ int lu_panel(Smem<T, PW>& s, int m, int kb, int* piv)
{
    const int tid = threadIdx.x;
    int zero = 0;
    // candidates of column 0
    float bv = -1.f;
    int bi = INT_MAX;
    for (int r = tid; r < m; r += T) {
        const float a = fabsf(s.P[r]);
        if (bi == INT_MAX || a > bv) { bv = a; bi = r; }
    }
    for (int j = 0; j < kb; ++j) {
        const int p = block_argmax<T>(bv, bi, s.rv, s.ri);  // barrier: column j final
        if (tid == 0) piv[j] = p;
        if (p != j && tid < kb) {
            const float t = s.P[tid * kLdp + j];
            s.P[tid * kLdp + j] = s.P[tid * kLdp + p];
            s.P[tid * kLdp + p] = t;
        }
        __syncthreads();
        const float pv = s.P[j * kLdp + j];
        if (pv == 0.f && zero == 0) zero = j + 1;
        const bool recip = fabsf(pv) >= FLT_MIN;
        const float rcp = 1.0f / pv;
        // scale column j, update columns j+1.. of the own rows, candidates of
        // column j+1 on the way
        bv = -1.f;
        bi = INT_MAX;
        for (int r = j + 1 + tid; r < m; r += T) {
            float l = s.P[j * kLdp + r];
            if (pv != 0.f) {
                l = recip ? l * rcp : l / pv;
                s.P[j * kLdp + r] = l;
            }
            for (int c = j + 1; c < kb; ++c)
                s.P[c * kLdp + r] = fmaf(-l, s.P[c * kLdp + j], s.P[c * kLdp + r]);
            if (j + 1 < kb) {
                const float a = fabsf(s.P[(j + 1) * kLdp + r]);
                if (bi == INT_MAX || a > bv) { bv = a; bi = r; }
            }
        }
    }
    __syncthreads();
    return zero;
}

// Cholesky of the m x kb panel P (diagonal block on top): the first failing
// column + 1, or 0.  Columns past a failure are left as they are.
template <int T, int PW>
__device__ int chol_panel(Smem<T, PW>& s, int m, int kb)
{
    const int tid = threadIdx.x;
    for (int j = 0; j < kb; ++j) {
        const float d = s.P[j * kLdp + j];  // final: updated before the last barrier
        if (!(d > 0.f)) return j + 1;       // uniform: every thread read the same value
        const float sd = sqrtf(d);
        const float rcp = 1.0f / sd;
        for (int r = j + 1 + tid; r < m; r += T) {
            const float l = s.P[j * kLdp + r] * rcp;
            s.P[j * kLdp + r] = l;
            if (r < kb) s.col[r] = l;
        }
        __syncthreads();
        if (tid == 0) s.P[j * kLdp + j] = sd;
        for (int r = j + 1 + tid; r < m; r += T) {
            const float l = s.P[j * kLdp + r];
            const int cmax = min(kb - 1, r);
            for (int c = j + 1; c <= cmax; ++c)
                s.P[c * kLdp + r] = fmaf(-l, s.col[c], s.P[c * kLdp + r]);
        }
        __syncthreads();
    }
    return 0;
}

// P (m x kb) <-> global A at the panel's top-left corner (element e is row
// e % m of column e / m: coalesced), eight loads in flight per thread.
template <int T, int PW, bool TO_SMEM>
__device__ __forceinline__ void move_panel(Smem<T, PW>& s, float* A, long long lda, int m, int kb)
{
    const int total = m * kb;
    int e = threadIdx.x;
    for (; e + 7 * T < total; e += 8 * T) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * T, c = q / m, r = q - c * m;
            v[u] = TO_SMEM ? A[(long long)c * lda + r] : s.P[c * kLdp + r];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int q = e + u * T, c = q / m, r = q - c * m;
            if (TO_SMEM) s.P[c * kLdp + r] = v[u];
            else A[(long long)c * lda + r] = v[u];
        }
    }
    for (; e < total; e += T) {
        const int c = e / m, r = e - c * m;
        if (TO_SMEM) s.P[c * kLdp + r] = A[(long long)c * lda + r];
        else A[(long long)c * lda + r] = s.P[c * kLdp + r];
    }
}

// --------------------------------------------------------- trailing update
// C(rows x cw) -= Aop(rows x kb) * Bop(kb x cw): Aop(r, q) = P[q * kLdp + a0 + r],
// Bop(q, c) = bsrc[q * bld + c], C(r, c) = C[c * ldc + r] in global memory.
// 8 x 4 register tiles: T/16 row groups x 16 column groups of 4 (64 columns);
// with `lower` only entries with r + diag >= c are written (diag: the offset
// of C's rows against its columns).  a0, bld and kb are multiples of 4.
template <int T, int PW>
__device__ __forceinline__ void update_chunk(const Smem<T, PW>& s, int a0, int rows, int kb,
                                             const float* bsrc, int bld, int cw, float* C,
                                             long long ldc, bool lower, int diag)
{
    constexpr int TY = T / 16;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int first = lower ? max(0, ((0 - diag) / 8) * 8) : 0;
    for (int rb = first; rb < rows; rb += TY * 8) {
        const int r = rb + ty * 8;
        if (r >= rows) continue;
        if (lower && r + 7 + diag < tx * 4) continue;  // tile wholly above the diagonal
        float acc[8][4] = {};
        const float* ap = s.P + a0 + r;
        for (int q = 0; q < kb; ++q) {
            const float4 x0 = *reinterpret_cast<const float4*>(ap + q * kLdp);
            const float4 x1 = *reinterpret_cast<const float4*>(ap + q * kLdp + 4);
            const float4 y = *reinterpret_cast<const float4*>(bsrc + q * bld + tx * 4);
            const float av[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
            const float bv[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(av[u], bv[v], acc[u][v]);
        }
        float old[8][4];  // every load of the tile before its first store
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int c = tx * 4 + v;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int rr = r + u;
                const bool ok = c < cw && rr < rows && (!lower || rr + diag >= c);
                old[u][v] = ok ? C[(long long)c * ldc + rr] : 0.f;
            }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int c = tx * 4 + v;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int rr = r + u;
                if (c < cw && rr < rows && (!lower || rr + diag >= c))
                    C[(long long)c * ldc + rr] = old[u][v] - acc[u][v];
            }
        }
    }
}

// ------------------------------------------------------------------ LU
template <int T, int PW>
__device__ int lu_factor(Smem<T, PW>& s, float* A, int n, long long lda, int* ipiv)
{
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    __shared__ int s_piv[PW];
    __shared__ int s_nm;
    int info = 0;
    for (int k = 0; k < n; k += PW) {
        const int kb = min(PW, n - k), m = n - k;
        float* Ak = A + (long long)k * lda + k;  // panel's top-left corner
        move_panel<T, PW, true>(s, Ak, lda, m, kb);
        __syncthreads();
        const int z = lu_panel<T, PW>(s, m, kb, s_piv);
        if (z && !info) info = k + z;
        move_panel<T, PW, false>(s, Ak, lda, m, kb);
        // compose the panel's interchanges into moves (panel rows)
        for (int r = tid; r < m; r += T) s.rowmap[r] = r;
        if (tid == 0) s_nm = 0;
        __syncthreads();
        if (tid == 0)
            for (int j = 0; j < kb; ++j) {
                const int p = s_piv[j];
                ipiv[k + j] = k + p + 1;
                const int t = s.rowmap[j];
                s.rowmap[j] = s.rowmap[p];
                s.rowmap[p] = t;
            }
        __syncthreads();
        if (tid < 2 * kb) {  // candidate rows j and piv[j]; the first occurrence adds its move
            const int t = tid < kb ? tid : s_piv[tid - kb];
            bool first = true;
            for (int q = 0; q < tid; ++q)
                if ((q < kb ? q : s_piv[q - kb]) == t) first = false;
            if (first && s.rowmap[t] != t) {
                const int q = atomicAdd(&s_nm, 1);
                s.mv[q] = s.rowmap[t];
                s.mv[2 * PW + q] = t;
            }
        }
        __syncthreads();
        const int nm = s_nm;
        // apply the moves to the columns left and right of the panel: one warp
        // per column, four columns per pass, every source of a column read
        // before any of its targets is written
        const int src0 = lane < nm ? s.mv[lane] : 0, src1 = lane + 32 < nm ? s.mv[lane + 32] : 0;
        const int tgt0 = lane < nm ? s.mv[2 * PW + lane] : 0;
        const int tgt1 = lane + 32 < nm ? s.mv[2 * PW + lane + 32] : 0;
        for (int c = warp; c < n - kb; c += 4 * (T / 32)) {
            float v0[4], v1[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int cu = c + u * (T / 32);
                v0[u] = v1[u] = 0.f;
                if (cu < n - kb) {
                    const float* Ac = A + (long long)(cu < k ? cu : cu + kb) * lda + k;
                    if (lane < nm) v0[u] = Ac[src0];
                    if (lane + 32 < nm) v1[u] = Ac[src1];
                }
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int cu = c + u * (T / 32);
                if (cu < n - kb) {
                    float* Ac = A + (long long)(cu < k ? cu : cu + kb) * lda + k;
                    if (lane < nm) Ac[tgt0] = v0[u];
                    if (lane + 32 < nm) Ac[tgt1] = v1[u];
                }
            }
        }
        __syncthreads();
        const int m2 = m - kb;  // trailing rows / columns
        // U12 = L11^{-1} A12 (unit lower) for every trailing column at once,
        // one thread per column
        for (int c = tid; c < m2; c += T) {
            float* colp = A + (long long)(k + kb + c) * lda + k;
            float xv[PW];
#pragma unroll
            for (int q = 0; q < PW; ++q) xv[q] = q < kb ? colp[q] : 0.f;
#pragma unroll
            for (int q = 0; q < PW; ++q)
#pragma unroll
                for (int r = q + 1; r < PW; ++r) xv[r] = fmaf(-s.P[q * kLdp + r], xv[q], xv[r]);
#pragma unroll
            for (int q = 0; q < PW; ++q)
                if (q < kb) colp[q] = xv[q];
        }
        __syncthreads();
        for (int c0 = 0; c0 < m2; c0 += kChunk) {
            const int cw = min(kChunk, m2 - c0);
            // the chunk's U12 block into shared memory, all loads in flight
            constexpr int kPer = (PW * kChunk + T - 1) / T;
            float v[kPer];
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int e = threadIdx.x + u * T, c = e / PW, q = e - c * PW;
                v[u] = (e < PW * kChunk && c < cw && q < kb)
                           ? A[(long long)(k + kb + c0 + c) * lda + k + q]
                           : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int e = threadIdx.x + u * T, c = e / PW, q = e - c * PW;
                if (e < PW * kChunk) s.Ub[q * kUbLd + c] = v[u];
            }
            __syncthreads();
            update_chunk<T, PW>(s, kb, m2, kb, s.Ub, kUbLd, cw,
                                A + (long long)(k + kb + c0) * lda + k + kb, lda, false, 0);
            __syncthreads();
        }
    }
    return info;
}

// ------------------------------------------------------------ Cholesky
template <int T, int PW>
__device__ int chol_factor(Smem<T, PW>& s, float* A, int n, long long lda)
{
    for (int k = 0; k < n; k += PW) {
        const int kb = min(PW, n - k), m = n - k;
        float* Ak = A + (long long)k * lda + k;
        move_panel<T, PW, true>(s, Ak, lda, m, kb);
        __syncthreads();
        const int f = chol_panel<T, PW>(s, m, kb);
        // write back the lower part (the strictly upper part of the diagonal
        // block keeps its input values)
        for (int c = 0; c < kb; ++c)
            for (int r = c + threadIdx.x; r < m; r += T) Ak[(long long)c * lda + r] = s.P[c * kLdp + r];
        if (f) {
            if (threadIdx.x == 0) {
                // the failing column's diagonal keeps the updated value, as xPOTRF
                Ak[(long long)(f - 1) * lda + f - 1] = s.P[(f - 1) * kLdp + f - 1];
            }
            __syncthreads();
            return k + f;
        }
        __syncthreads();
        const int m2 = m - kb;
        for (int c0 = 0; c0 < m2; c0 += kChunk) {
            const int cw = min(kChunk, m2 - c0);
            // rows c0.. of the trailing block, columns c0 .. c0+cw, lower part
            update_chunk<T, PW>(s, kb + c0, m2 - c0, kb, s.P + kb + c0, kLdp, cw,
                                A + (long long)(k + kb + c0) * lda + k + kb + c0, lda, true, 0);
        }
        __syncthreads();
    }
    return 0;
}

// ------------------------------------------------------------------ solves
// Blocked substitutions on x (shared memory): warp 0 solves each PW x PW
// diagonal block with shuffles (the block's entries prefetched into
// registers), then all threads update the remaining rows with the block's
// columns (coalesced column reads).

// x <- L^{-1} x, L lower (unit diagonal when `unit`), column-major in A.
template <int T, int PW>
__device__ void forward_lower(const float* A, int n, long long lda, float* x, bool unit)
{
    const int tid = threadIdx.x, lane = tid & 31;
    for (int k = 0; k < n; k += PW) {
        const int kb = min(PW, n - k);
        if (tid < 32) {
            for (int h = 0; h < PW; h += 32) {  // PW <= 32: one pass
                const int i = h + lane;
                float li[PW];
#pragma unroll
                for (int q = 0; q < PW; ++q)
                    li[q] = (i < kb && q <= i && q < kb) ? A[(long long)(k + q) * lda + k + i] : 0.f;
                float xi = i < kb ? x[k + i] : 0.f;
#pragma unroll
                for (int q = 0; q < PW; ++q) {
                    if (q < kb) {
                        if (!unit && i == q) xi = xi / li[q];
                        const float xq = __shfl_sync(0xffffffffu, xi, q);
                        if (i > q) xi = fmaf(-li[q], xq, xi);
                    }
                }
                if (i < kb) x[k + i] = xi;
            }
        }
        __syncthreads();
        for (int r = k + kb + tid; r < n; r += T) {
            float a[PW];  // the row's block entries, all loads in flight together
#pragma unroll
            for (int q = 0; q < PW; ++q) a[q] = q < kb ? A[(long long)(k + q) * lda + r] : 0.f;
            float acc = x[r];
#pragma unroll
            for (int q = 0; q < PW; ++q)
                if (q < kb) acc = fmaf(-a[q], x[k + q], acc);
            x[r] = acc;
        }
        __syncthreads();
    }
}

// x <- U^{-1} x, U the upper triangle of A (non-unit).
template <int T, int PW>
__device__ void backward_upper(const float* A, int n, long long lda, float* x)
{
    const int tid = threadIdx.x, lane = tid & 31;
    const int nblk = (n + PW - 1) / PW;
    for (int bi = nblk - 1; bi >= 0; --bi) {
        const int k = bi * PW, kb = min(PW, n - k);
        if (tid < 32) {
            const int i = lane;
            float ui[PW];
#pragma unroll
            for (int q = 0; q < PW; ++q)
                ui[q] = (i < kb && q >= i && q < kb) ? A[(long long)(k + q) * lda + k + i] : 0.f;
            float xi = i < kb ? x[k + i] : 0.f;
#pragma unroll
            for (int q = PW - 1; q >= 0; --q) {
                if (q < kb) {
                    if (i == q) xi = xi / ui[q];
                    const float xq = __shfl_sync(0xffffffffu, xi, q);
                    if (i < q) xi = fmaf(-ui[q], xq, xi);
                }
            }
            if (i < kb) x[k + i] = xi;
        }
        __syncthreads();
        for (int r = tid; r < k; r += T) {
            float a[PW];  // the row's block entries, all loads in flight together
#pragma unroll
            for (int q = 0; q < PW; ++q) a[q] = q < kb ? A[(long long)(k + q) * lda + r] : 0.f;
            float acc = x[r];
#pragma unroll
            for (int q = 0; q < PW; ++q)
                if (q < kb) acc = fmaf(-a[q], x[k + q], acc);
            x[r] = acc;
        }
        __syncthreads();
    }
}

// x <- L^{-T} x, L lower (non-unit): per block, the dot products of the
// block's columns with the already solved rows below (one warp per column),
// then the block backward on warp 0.
template <int T, int PW>
__device__ void backward_lower_t(const float* A, int n, long long lda, float* x, float* dots)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nblk = (n + PW - 1) / PW;
    for (int bi = nblk - 1; bi >= 0; --bi) {
        const int k = bi * PW, kb = min(PW, n - k);
        for (int j = warp; j < kb; j += T / 32) {
            const float* cj = A + (long long)(k + j) * lda;
            float sum = 0.f;
#pragma unroll 4
            for (int r = k + kb + lane; r < n; r += 32) sum = fmaf(cj[r], x[r], sum);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
            if (lane == 0) dots[j] = sum;
        }
        __syncthreads();
        if (tid < 32) {
            const int i = lane;
            float li[PW];  // L(k + q, k + i), q >= i: column k + i of the block
#pragma unroll
            for (int q = 0; q < PW; ++q)
                li[q] = (i < kb && q >= i && q < kb) ? A[(long long)(k + i) * lda + k + q] : 0.f;
            float xi = i < kb ? x[k + i] - dots[i] : 0.f;
#pragma unroll
            for (int q = PW - 1; q >= 0; --q) {
                if (q < kb) {
                    if (i == q) xi = xi / li[q];
                    const float xq = __shfl_sync(0xffffffffu, xi, q);
                    if (i < q) xi = fmaf(-li[q], xq, xi);
                }
            }
            if (i < kb) x[k + i] = xi;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ kernel
// Register budget for two CTAs per SM at 256 threads and three at 128 (the
// 16-column panel's shared footprint allows three): one matrix per CTA spends
// much of its time at barriers, so co-resident CTAs fill the gaps.
template <int T>
constexpr int min_ctas() { return T >= 512 ? 1 : (T >= 256 ? 2 : 3); }

template <int T, int PW>
__global__ void __launch_bounds__(T, min_ctas<T>()) batched_factor_solve_kernel(BatchArgs a)
{
    extern __shared__ __align__(16) float sm[];
    Smem<T, PW> s(sm);
    __shared__ int s_item;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = (int)atomicAdd(a.queue, 1u);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= a.count) break;
        const int idx = a.order[it];
        const int n = a.n[idx];
        const int op = a.op[idx];
        if (n <= 0 || (op == 0 && n > kMaxChol) || (op != 0 && n > kMaxLu)) continue;
        float* A = a.A[idx];
        const long long lda = a.lda[idx];
        float* b = a.b[idx];
        int info;
        if (op == 0) info = chol_factor<T, PW>(s, A, n, lda);
        else info = lu_factor<T, PW>(s, A, n, lda, a.ipiv[idx]);
        if (tid == 0) a.info[idx] = info;
        if (info) continue;
        // solve: x = b (LU: with the row interchanges applied in order)
        for (int r = tid; r < n; r += T) s.x[r] = b[r];
        __syncthreads();
        if (op != 0) {
            if (tid == 0) {
                const int* ip = a.ipiv[idx];
                for (int i = 0; i < n; ++i) {
                    const int p = ip[i] - 1;
                    if (p != i) {
                        const float t = s.x[i];
                        s.x[i] = s.x[p];
                        s.x[p] = t;
                    }
                }
            }
            __syncthreads();
            forward_lower<T, PW>(A, n, lda, s.x, true);
            backward_upper<T, PW>(A, n, lda, s.x);
        } else {
            forward_lower<T, PW>(A, n, lda, s.x, false);
            backward_lower_t<T, PW>(A, n, lda, s.x, s.col);
        }
        for (int r = tid; r < n; r += T) b[r] = s.x[r];
        __syncthreads();
    }
}

// Launch shapes: threads per CTA and panel width.
struct Variant {
    int threads, panel;
};
constexpr Variant kVariants[] = {{128, 32}, {256, 32}, {512, 32}, {128, 16}, {256, 16}, {512, 16}};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));

template <int T, int PW>
hdbf_status launch_batched(hdbf_context* ctx, const BatchArgs& a)
{
    const size_t smem = smem_floats<PW>() * sizeof(float);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batched_factor_solve_kernel<T, PW>,
                                                      T, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const int ctas = std::max(1, std::min(a.count, ctx->sm_count * per_sm));
    batched_factor_solve_kernel<T, PW><<<ctas, T, smem, ctx->stream>>>(a);
    ctx->launches++;
    return last_cuda(ctx);
}

template <int T, int PW>
void configure_one()
{
    cudaFuncSetAttribute(batched_factor_solve_kernel<T, PW>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(smem_floats<PW>() * sizeof(float)));
}

}  // namespace

void configure_batched_kernels(hdbf_context* ctx)
{
    (void)ctx;
    configure_one<128, 32>();
    configure_one<256, 32>();
    configure_one<512, 32>();
    configure_one<128, 16>();
    configure_one<256, 16>();
    configure_one<512, 16>();
    cudaGetLastError();
}

}  // namespace hdbf

using namespace hdbf;

extern "C" {

int hdbf_batched_num_variants(void) { return kNumVariants; }

hdbf_status hdbf_batched_variant_shape(int variant, int* threads, int* panel)
{
    if (variant < 0 || variant >= kNumVariants || !threads || !panel)
        return HDBF_STATUS_INVALID_VALUE;
    *threads = kVariants[variant].threads;
    *panel = kVariants[variant].panel;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_batched_factor_solve(hdbf_handle h, int variant, int count, const int* order,
                                      const int* op, const int* n, const int* lda, float* const* A,
                                      float* const* b, int* const* ipiv, int* info,
                                      unsigned int* queue)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (count < 0 || variant < 0 || variant >= kNumVariants)
        return h->last_status = HDBF_STATUS_INVALID_VALUE;
    if (count == 0) return h->last_status = HDBF_STATUS_SUCCESS;
    if (!order || !op || !n || !lda || !A || !b || !ipiv || !info || !queue)
        return h->last_status = HDBF_STATUS_INVALID_VALUE;
    BatchArgs a{count, order, op, n, lda, A, b, ipiv, info, queue};
    const std::vector<long long> key = {41, variant, count, (long long)order, (long long)op,
                                        (long long)n, (long long)lda, (long long)A, (long long)b,
                                        (long long)ipiv, (long long)info, (long long)queue};
    return h->last_status = run_graph(h, key, [&]() -> hdbf_status {
        cudaMemsetAsync(queue, 0, sizeof(unsigned int), h->stream);
        ProfScope prof(h, kClsBatched, 0.0, 0.0);
        switch (variant) {
        case 0: return launch_batched<128, 32>(h, a);
        case 1: return launch_batched<256, 32>(h, a);
        case 2: return launch_batched<512, 32>(h, a);
        case 3: return launch_batched<128, 16>(h, a);
        case 4: return launch_batched<256, 16>(h, a);
        default: return launch_batched<512, 16>(h, a);
        }
    });
}

}  // extern "C"
