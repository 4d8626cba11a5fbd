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

// ------------------------------------------------- diagonal tile: L and L^-1
// The nb x nb (nb <= 64) lower tile at T is factored and inverted by the
// whole CTA in four 16-column blocks (shared memory S = tile, X = inverse,
// both row-major with pitch kP; identity padding beyond nb):
//   for each block: warp 0 factors the 16 x 16 diagonal block with
//   shuffles (lane = row) and inverts it (lane = column); all threads solve
//   the rows below against that inverse (L_r = A_r X_d^T) and apply the
//   rank-16 update to the trailing lower triangle;
// then L^-1 by recursive doubling, 16 -> 32 -> 64:
//   X21 = -X22 (L21 X11).
// Twelve barriers for the factorization, eight for the inverse, instead of a
// barrier (or two) per column.
constexpr int kP = 65;   // row pitch of S and X (odd: conflict-free rows and columns)
constexpr int kDB = 16;  // diagonal block

// Warp 0: Cholesky of the 16 x 16 diagonal block at (c0, c0) of S and its
// inverse into X; returns the first failing column of the block or -1.
__device__ int chol16_inv16(float* S, float* X, int c0)
{
    const int l = threadIdx.x & 31;
    const int lr = l < kDB ? l : 0;  // lanes 16..31 mirror lane 0 (results unused)
    float v[kDB];
#pragma unroll
    for (int m = 0; m < kDB; ++m) v[m] = m <= lr ? S[(c0 + lr) * kP + c0 + m] : 0.f;
    int fail = -1;
#pragma unroll
    for (int j = 0; j < kDB; ++j) {
        const float dj = __shfl_sync(0xffffffffu, v[j], j);
        if (!(dj > 0.f)) {  // uniform in the warp
            fail = j;
            break;
        }
        const float sd = sqrtf(dj);
        const float rcp = 1.0f / sd;
        if (lr == j) v[j] = sd;
        else if (lr > j) v[j] = v[j] * rcp;
#pragma unroll
        for (int c = j + 1; c < kDB; ++c) {
            const float lc = __shfl_sync(0xffffffffu, v[j], c);
            if (lr >= c) v[c] = fmaf(-v[j], lc, v[c]);
        }
    }
    if (l < kDB) {
#pragma unroll
        for (int m = 0; m < kDB; ++m)
            if (m <= l) S[(c0 + l) * kP + c0 + m] = v[m];
    }
    if (fail >= 0) return fail;
    // inverse: lane t solves L x = e_t (column t of X_d), L(i, m) from lane i
    const int t = lr;
    float x[kDB];
#pragma unroll
    for (int i = 0; i < kDB; ++i) {
        float acc = (i == t) ? 1.f : 0.f;
#pragma unroll
        for (int m = 0; m < i; ++m) acc = fmaf(-__shfl_sync(0xffffffffu, v[m], i), x[m], acc);
        x[i] = acc / __shfl_sync(0xffffffffu, v[i], i);
    }
    if (l < kDB) {
#pragma unroll
        for (int i = 0; i < kDB; ++i) X[(c0 + i) * kP + c0 + l] = x[i];
    }
    return -1;
}

// Factor the tile at T (nb <= 64) into S (lower, row-major pitch kP) and
// invert it into X; L goes back to T and L^-1 (zero above the diagonal,
// identity beyond nb) to D (column-major, leading dimension 64).  Returns the
// first failing column or -1 (uniform over the CTA); on failure T holds the
// partial factor and D is not written.
__device__ int factor_invert_tile(float* T, long long ld, int nb, float* S, float* X, float* D,
                                  int* s_fail)
{
    const int tid = threadIdx.x;
    {
        float vv[kT * kT / kThreads];
#pragma unroll
        for (int u = 0; u < kT * kT / kThreads; ++u) {
            const int q = tid + u * kThreads, c = q >> 6, r = q & 63;
            vv[u] = (r < nb && c < nb && r >= c) ? __ldcg(T + (long long)c * ld + r)
                                                 : (r == c ? 1.f : 0.f);
        }
#pragma unroll
        for (int u = 0; u < kT * kT / kThreads; ++u) {
            const int q = tid + u * kThreads, c = q >> 6, r = q & 63;
            S[r * kP + c] = vv[u];
            X[r * kP + c] = 0.f;
        }
    }
    if (tid == 0) *s_fail = -1;
    __syncthreads();
    for (int kb = 0; kb < kT / kDB; ++kb) {
        const int c0 = kb * kDB;
        if (tid < 32) {
            const int f = chol16_inv16(S, X, c0);
            if (tid == 0 && f >= 0) *s_fail = c0 + f;
        }
        __syncthreads();
        if (*s_fail >= 0) break;
        const int rows = kT - c0 - kDB;  // rows below the block
        if (rows > 0) {
            // L_r = A_r X_d^T for rows r below: thread = (row, 4 columns)
            const int r = c0 + kDB + (tid >> 2), g = tid & 3;
            float out[4] = {0.f, 0.f, 0.f, 0.f};
            if (tid < rows * 4) {
                float a[kDB];
#pragma unroll
                for (int m = 0; m < kDB; ++m) a[m] = S[r * kP + c0 + m];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    const int j = g * 4 + jj;
#pragma unroll
                    for (int m = 0; m < kDB; ++m)
                        if (m <= j) out[jj] = fmaf(a[m], X[(c0 + j) * kP + c0 + m], out[jj]);
                }
            }
            __syncthreads();
            if (tid < rows * 4) {
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) S[r * kP + c0 + g * 4 + jj] = out[jj];
            }
            __syncthreads();
            // trailing lower triangle: S(r, c) -= sum_m L(r, c0+m) L(c, c0+m)
            for (int idx = tid; idx < rows * rows; idx += kThreads) {
                const int rr = idx / rows, cc = idx - rr * rows;
                if (cc > rr) continue;
                const int r2 = c0 + kDB + rr, c2 = c0 + kDB + cc;
                float acc = S[r2 * kP + c2];
#pragma unroll
                for (int m = 0; m < kDB; ++m)
                    acc = fmaf(-S[r2 * kP + c0 + m], S[c2 * kP + c0 + m], acc);
                S[r2 * kP + c2] = acc;
            }
            __syncthreads();
        }
    }
    const int fail = *s_fail;
    // L back to T (lower part inside nb x nb)
#pragma unroll
    for (int u = 0; u < kT * kT / kThreads; ++u) {
        const int q = tid + u * kThreads, c = q >> 6, r = q & 63;
        if (r < nb && c < nb && r >= c) T[(long long)c * ld + r] = S[r * kP + c];
    }
    if (fail >= 0) return fail;
    // L^-1 by recursive doubling: for sibling blocks of size h at b0 and
    // b0 + h, X21 = -X22 (L21 X11); T21 = L21 X11 is kept in the X21 slot.
    for (int h = kDB; h < kT; h *= 2) {
        const int pairs = kT / (2 * h);
        const int outs = pairs * h * h;  // outputs per phase
        const int per = (outs + kThreads - 1) / kThreads;  // <= 4
        float o[4];
        // phase a: T21(i, j) = sum_{m >= j} L21(i, m) X11(m, j)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            o[u] = 0.f;
            const int q = tid + u * kThreads;
            if (u < per && q < outs) {
                const int pr = q / (h * h), e = q - pr * h * h, i = e / h, j = e - i * h;
                const int b0 = pr * 2 * h;
                float acc = 0.f;
                for (int m = j; m < h; ++m)
                    acc = fmaf(S[(b0 + h + i) * kP + b0 + m], X[(b0 + m) * kP + b0 + j], acc);
                o[u] = acc;
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int q = tid + u * kThreads;
            if (u < per && q < outs) {
                const int pr = q / (h * h), e = q - pr * h * h, i = e / h, j = e - i * h;
                const int b0 = pr * 2 * h;
                X[(b0 + h + i) * kP + b0 + j] = o[u];
            }
        }
        __syncthreads();
        // phase b: X21(i, j) = -sum_{m <= i} X22(i, m) T21(m, j)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            o[u] = 0.f;
            const int q = tid + u * kThreads;
            if (u < per && q < outs) {
                const int pr = q / (h * h), e = q - pr * h * h, i = e / h, j = e - i * h;
                const int b0 = pr * 2 * h;
                float acc = 0.f;
                for (int m = 0; m <= i; ++m)
                    acc = fmaf(X[(b0 + h + i) * kP + b0 + h + m], X[(b0 + h + m) * kP + b0 + j],
                               acc);
                o[u] = -acc;
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int q = tid + u * kThreads;
            if (u < per && q < outs) {
                const int pr = q / (h * h), e = q - pr * h * h, i = e / h, j = e - i * h;
                const int b0 = pr * 2 * h;
                X[(b0 + h + i) * kP + b0 + j] = o[u];
            }
        }
        __syncthreads();
    }
    // D (column-major, 64 x 64) = X
#pragma unroll
    for (int u = 0; u < kT * kT / kThreads; ++u) {
        const int q = tid + u * kThreads, c = q >> 6, r = q & 63;
        D[q] = X[r * kP + c];
    }
    __syncthreads();
    return -1;
}

__global__ void __launch_bounds__(kThreads, 1)
potrf_block_kernel(int n, float* A, long long lda, int* info, int info_base, float* W,
                   long long ldw, float* dinv, float* Tsc, unsigned* ctr, int* fail,
                   int* abort_flag, int* err, const int* run_if)
{
    __shared__ __align__(16) float As[kT * kLdS];
    __shared__ __align__(16) float Bs[kT * kLdS];
    __shared__ int s_tile_fail;
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
        const int f = factor_invert_tile(tile(k, k), lda, ext(k), As, Bs,
                                         dinv + (long long)k * kT * kT, &s_tile_fail);
        if (f >= 0) {
            if (tid == 0) {
                if (info) atomicCAS(info, 0, info_base + k * kT + f + 1);
                atomicExch(fail, 1);
            }
            return false;
        }
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
