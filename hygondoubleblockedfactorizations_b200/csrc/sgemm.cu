// FP32 SIMT trailing-update GEMM / SYRK:  C -= op(A) * op(B).
//
// Replaces the reference's rocblas_sgemm (N,T) and (N,N) update calls
// (src/gemm/update_gemm.cpp:29-44, src/getrf/getrf_npvt_internal.h:109-124)
// and rocblas_ssyrk lower (src/syrk/kblocked_syrk.cpp:33-45); the (T,N) form
// serves the transposed-factor back substitution of the solves.
//
// Design: 128x128 CTA tile, K-step 8, 256 threads each owning an 8x8
// register micro-tile (two 4-row x two 4-column quads, so the shared-memory
// fragment reads are float4 broadcasts), double-buffered shared memory fed
// from a register prefetch of the next K-slab, one __syncthreads per slab.
// Two CTAs per SM (<= 128 registers per thread).  Every product is an IEEE
// FP32 FFMA; accumulation runs in k order from zero, then C - acc.
#include <algorithm>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int BM = 128;
constexpr int BN = 128;
constexpr int BK = 8;
constexpr int NTHR = 256;

// Operand forms: C -= A * B^T (NT: A is M x K, B is N x K), C -= A * B (NN: B
// is K x N), C -= A^T * B (TN: A is K x M, B is K x N).  All column-major.
enum Mode { kNT = 0, kNN = 1, kTN = 2 };

template <bool VEC>
__device__ __forceinline__ float4 load_col4(const float* p, int row, int rows_valid)
{
    // Four consecutive rows of one column; rows beyond rows_valid read 0.
    float4 v;
    if (VEC && row + 3 < rows_valid) {
        v = __ldg(reinterpret_cast<const float4*>(p));
    } else {
        v.x = (row + 0 < rows_valid) ? __ldg(p + 0) : 0.f;
        v.y = (row + 1 < rows_valid) ? __ldg(p + 1) : 0.f;
        v.z = (row + 2 < rows_valid) ? __ldg(p + 2) : 0.f;
        v.w = (row + 3 < rows_valid) ? __ldg(p + 3) : 0.f;
    }
    return v;
}

template <int MODE, bool VEC, bool TRI, bool SPLIT>
__global__ void __launch_bounds__(NTHR, 2)
sgemm_sub_kernel(int M, int N, int K, const float* __restrict__ A, long long lda,
                 const float* __restrict__ B, long long ldb, float* __restrict__ C,
                 long long ldc, int tiles_m, const int* __restrict__ run_if,
                 float* __restrict__ part, int kc, int tiles)
{
    if (run_if && *run_if == 0) return;  // conditional launch (RunIf) not taken
    constexpr bool AT = MODE == kTN;  // A read k-contiguous (transposed load)
    constexpr bool BT = MODE != kNT;  // B read k-contiguous (transposed load)
    // Split K (part != nullptr): CTA blockIdx.x handles K chunk s of tile
    // blockIdx.x - s * tiles and stores its partial product, from zero, in
    // part[s] (M x N, leading dimension M); split_reduce_kernel applies them.
    int bid = blockIdx.x;
    int split = 0;
    if (SPLIT) {
        split = bid / tiles;
        bid -= split * tiles;
        const int k0 = split * kc;
        K = min(kc, K - k0);
        A += AT ? (long long)k0 : (long long)k0 * lda;
        B += BT ? (long long)k0 : (long long)k0 * ldb;
    }
    const int tm = bid % tiles_m;
    const int tn = bid / tiles_m;
    const int m0 = tm * BM;
    const int n0 = tn * BN;
    if (TRI && m0 + BM <= n0) return;  // tile strictly above the diagonal

    constexpr int ASTR = AT ? BM + 4 : BM;  // pad breaks STS bank conflicts
    constexpr int BSTR = BT ? BN + 4 : BN;
    __shared__ __align__(16) float As[2][BK][ASTR];
    __shared__ __align__(16) float Bs[2][BK][BSTR];

    const int tid = threadIdx.x;
    // k-contiguous operands: a thread loads 4 consecutive k of one row/column
    // (index t>>1, k offset (t&1)*4); mn-contiguous operands: 4 consecutive
    // rows of one k column ((t&31)*4, t>>5).
    const int ak = AT ? (tid & 1) * 4 : (tid >> 5);
    const int am = AT ? (tid >> 1) : (tid & 31) * 4;
    const int bk = BT ? (tid & 1) * 4 : (tid >> 5);
    const int bn = BT ? (tid >> 1) : (tid & 31) * 4;

    const float* a_ptr =
        AT ? A + (long long)(m0 + am) * lda + ak : A + (long long)ak * lda + (m0 + am);
    const float* b_ptr =
        BT ? B + (long long)(n0 + bn) * ldb + bk : B + (long long)bk * ldb + (n0 + bn);
    const long long a_step = AT ? (long long)BK : (long long)BK * lda;
    const long long b_step = BT ? (long long)BK : (long long)BK * ldb;

    auto fetch_a = [&](int k0) -> float4 {
        if (AT) {
            if (m0 + am < M) return load_col4<VEC>(a_ptr, k0 + ak, K);
            return make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (k0 + ak < K) return load_col4<VEC>(a_ptr, m0 + am, M);
        return make_float4(0.f, 0.f, 0.f, 0.f);
    };
    auto fetch_b = [&](int k0) -> float4 {
        if (BT) {
            if (n0 + bn < N) return load_col4<VEC>(b_ptr, k0 + bk, K);
            return make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (k0 + bk < K) return load_col4<VEC>(b_ptr, n0 + bn, N);
        return make_float4(0.f, 0.f, 0.f, 0.f);
    };
    auto stash = [&](int buf, float4 ra, float4 rb) {
        if (AT) {
            As[buf][ak + 0][am] = ra.x;
            As[buf][ak + 1][am] = ra.y;
            As[buf][ak + 2][am] = ra.z;
            As[buf][ak + 3][am] = ra.w;
        } else {
            *reinterpret_cast<float4*>(&As[buf][ak][am]) = ra;
        }
        if (BT) {
            Bs[buf][bk + 0][bn] = rb.x;
            Bs[buf][bk + 1][bn] = rb.y;
            Bs[buf][bk + 2][bn] = rb.z;
            Bs[buf][bk + 3][bn] = rb.w;
        } else {
            *reinterpret_cast<float4*>(&Bs[buf][bk][bn]) = rb;
        }
    };

    // 16 x 16 thread tiles; each warp covers 8 (ty) x 4 (tx) of them, so a
    // k-step's A and B fragment reads are one shared-memory wavefront each.
    const int tx = ((tid >> 5) & 3) * 4 + (tid & 3);
    const int ty = (tid >> 7) * 8 + ((tid & 31) >> 2);

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;

    auto slab = [&](int buf) {
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][64 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
    };

    const int ktiles = (K + BK - 1) / BK;
    // Interior tiles (the bulk of a large update): every operand quad is in
    // range, so the slab loads carry no bounds tests -- this kernel is
    // issue-bound, and the tests cost a tenth of its rate.
    const bool interior = VEC && m0 + BM <= M && n0 + BN <= N && (K % BK) == 0;
    if (interior) {
        float4 ra = __ldg(reinterpret_cast<const float4*>(a_ptr));
        float4 rb = __ldg(reinterpret_cast<const float4*>(b_ptr));
        stash(0, ra, rb);
        __syncthreads();
        int buf = 0;
        for (int kt = 0; kt < ktiles; ++kt) {
            const bool more = kt + 1 < ktiles;
            if (more) {
                a_ptr += a_step;
                b_ptr += b_step;
                ra = __ldg(reinterpret_cast<const float4*>(a_ptr));
                rb = __ldg(reinterpret_cast<const float4*>(b_ptr));
            }
            slab(buf);
            if (more) stash(buf ^ 1, ra, rb);
            __syncthreads();
            buf ^= 1;
        }
    } else {
        float4 ra = fetch_a(0);
        float4 rb = fetch_b(0);
        stash(0, ra, rb);
        __syncthreads();
        int buf = 0;
        for (int kt = 0; kt < ktiles; ++kt) {
            const bool more = kt + 1 < ktiles;
            if (more) {
                a_ptr += a_step;
                b_ptr += b_step;
                ra = fetch_a((kt + 1) * BK);
                rb = fetch_b((kt + 1) * BK);
            }
            slab(buf);
            if (more) stash(buf ^ 1, ra, rb);
            __syncthreads();
            buf ^= 1;
        }
    }

    const bool full_rows = (m0 + BM <= M);
    const bool full_cols = (n0 + BN <= N);
    if (SPLIT) {  // split K: store the partial product
        float* P = part + (long long)split * M * N;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int col = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
            if (col >= N) continue;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int row = m0 + h * 64 + ty * 4;
                float* pp = P + (long long)col * M + row;
                if (full_rows && (M & 3) == 0) {
                    *reinterpret_cast<float4*>(pp) = make_float4(
                        acc[h * 4 + 0][j], acc[h * 4 + 1][j], acc[h * 4 + 2][j], acc[h * 4 + 3][j]);
                } else {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (row + i < M) pp[i] = acc[h * 4 + i][j];
                }
            }
        }
        return;
    }
    // Epilogue: C -= acc.  Full interior tiles read all 16 C quads before
    // writing any (independent loads in flight together).
    const bool below_diag = !TRI || (m0 >= n0 + BN);
    if (VEC && full_rows && full_cols && below_diag) {
        float4 cq[8][2];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int col = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
#pragma unroll
            for (int h = 0; h < 2; ++h)
                cq[j][h] = __ldcg(reinterpret_cast<const float4*>(C + (long long)col * ldc + m0 +
                                                                  h * 64 + ty * 4));
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int col = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float4 c = cq[j][h];
                c.x -= acc[h * 4 + 0][j];
                c.y -= acc[h * 4 + 1][j];
                c.z -= acc[h * 4 + 2][j];
                c.w -= acc[h * 4 + 3][j];
                *reinterpret_cast<float4*>(C + (long long)col * ldc + m0 + h * 64 + ty * 4) = c;
            }
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int col = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
        if (col >= N) continue;
        float* cp = C + (long long)col * ldc;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int row = m0 + h * 64 + ty * 4;
            {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = row + i;
                    if (r < M && (!TRI || r >= col)) cp[r] -= acc[h * 4 + i][j];
                }
            }
        }
    }
}

// C -= sum over s of part[s] (in s order), lower triangle only when TRI.
template <bool TRI>
__global__ void split_reduce_kernel(int M, int N, int S, const float* __restrict__ part,
                                    float* __restrict__ C, long long ldc)
{
    const long long total = (long long)M * N;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int col = (int)(e / M), row = (int)(e - (long long)col * M);
        if (TRI && row < col) continue;
        float acc = part[e];
        for (int s = 1; s < S; ++s) acc += part[(long long)s * total + e];
        float* c = C + (long long)col * ldc + row;
        *c -= acc;
    }
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <int MODE, bool VEC, bool TRI>
void launch_sub(cudaStream_t s, int M, int N, int K, const float* A, long long lda,
                const float* B, long long ldb, float* C, long long ldc, const int* run_if,
                float* part = nullptr, int splits = 1, int kc = 0)
{
    const int tiles_m = (M + BM - 1) / BM;
    const int tiles_n = (N + BN - 1) / BN;
    const long long tiles = (long long)tiles_m * tiles_n;
    if (!part) {
        sgemm_sub_kernel<MODE, VEC, TRI, false><<<(unsigned)tiles, NTHR, 0, s>>>(
            M, N, K, A, lda, B, ldb, C, ldc, tiles_m, run_if, nullptr, 0, (int)tiles);
    } else {
        sgemm_sub_kernel<MODE, VEC, TRI, true><<<(unsigned)(tiles * splits), NTHR, 0, s>>>(
            M, N, K, A, lda, B, ldb, C, ldc, tiles_m, run_if, part, kc, (int)tiles);
        const long long total = (long long)M * N;
        const int g = (int)std::min<long long>((total + 255) / 256, 1184);
        split_reduce_kernel<TRI><<<g, 256, 0, s>>>(M, N, splits, part, C, ldc);
    }
}

}  // namespace

// K split against wave quantisation: a launch whose last wave of CTAs would
// leave SMs idle splits K into S chunks of whole K steps (at most 8, at least
// 512 K each, 256 under one wave) when that shortens the wave-model time ceil(tiles S / slots)
// x K / S (slots = two CTAs per SM) by at least 5% after a 3% charge per
// extra chunk for the ordered reduction of the partial products, which must
// fit in the scratch half; 1 = no split.
int split_count(const hdbf_context* ctx, int M, int N, int K, bool tri, int* kc)
{
    if (!ctx->ws || ctx->run_if) return 1;
    if (ctx->split_kc >= 0) {  // the plan of a whole GEMM this launch is a part of
        if (ctx->split_kc == 0) return 1;
        *kc = ctx->split_kc;
        const int S = (K + *kc - 1) / *kc;
        return (S > 1 && (long long)S * M * N <= (long long)kSplitFloats) ? S : 1;
    }
    if (K < 512) return 1;
    const long long tm = (M + BM - 1) / BM, tn = (N + BN - 1) / BN;
    long long tiles = tm * tn;
    if (tri) {  // tiles on or below the diagonal
        tiles = 0;
        for (long long j = 0; j < tn; ++j) tiles += std::max<long long>(0, tm - j);
    }
    if (tiles <= 0) return 1;
    const long long slots = 2LL * ctx->sm_count;
    auto chunk = [&](int S) { return ((K + S - 1) / S + BK - 1) / BK * BK; };
    auto cost = [&](int S) {
        const int c = chunk(S);
        const int parts = (K + c - 1) / c;
        const long long waves = (tiles * parts + slots - 1) / slots;
        return (double)waves * c * (1.0 + 0.03 * (parts - 1));
    };
    int best = 1;
    double best_cost = cost(1);
    for (int S = 2; S <= 8; ++S) {
        // chunks of at least 512 K (256 when the launch fills under a wave)
        if (K / S < (tiles < slots ? 256 : 512) || (long long)S * M * N > (long long)kSplitFloats)
            break;
        const double c = cost(S);
        if (c < 0.95 * best_cost) {
            best = S;
            best_cost = c;
        }
    }
    if (best < 2) return 1;
    *kc = chunk(best);
    return (K + *kc - 1) / *kc;
}

namespace {

hdbf_status sgemm_launch(hdbf_context* ctx, int mode, bool lower_only, int M, int N, int K,
                         const float* A, long long lda, const float* B, long long ldb, float* C,
                         long long ldc)
{
    if (M <= 0 || N <= 0 || K <= 0) return HDBF_STATUS_SUCCESS;
    if (!A || !B || !C) return HDBF_STATUS_INVALID_VALUE;
    if (lower_only && mode != kNT) return HDBF_STATUS_INVALID_VALUE;
    if (!lower_only && !ctx->no_skinny && !ctx->run_if && N <= 32 && M >= 4 * N && M >= 256)
        return sgemm_skinny(ctx, mode == kNT ? 0 : mode == kNN ? 1 : 2, M, N, K, A, lda, B, ldb,
                            C, ldc);
    const long long tiles = (long long)((M + BM - 1) / BM) * ((N + BN - 1) / BN);
    if (tiles > 0x7fffffffLL) return HDBF_STATUS_NOT_SUPPORTED;
    const bool vec = aligned16(A) && aligned16(B) && aligned16(C) && (lda % 4 == 0) &&
                     (ldb % 4 == 0) && (ldc % 4 == 0);
    cudaStream_t s = ctx->stream;
    const int* ri = ctx->run_if;
    double flops = 2.0 * (double)M * N * K;
    if (lower_only) {
        // only entries with row >= col: sum over cols j < min(M,N) of (M - j)
        const double d = (double)(M < N ? M : N);
        flops = 2.0 * (double)K * (d * (double)M - d * (d - 1.0) / 2.0);
    }
    ProfScope prof(ctx, kClsGemm, flops, 4.0 * ((double)M * K + (double)N * K + 2.0 * M * N), M,
                   N, K);
    int kc = 0;
    const int S = split_count(ctx, M, N, K, lower_only, &kc);
    float* part = S > 1 ? ws_split(ctx) : nullptr;
#define HDBF_SUB(MD, V, T) launch_sub<MD, V, T>(s, M, N, K, A, lda, B, ldb, C, ldc, ri, part, S, kc)
    if (mode == kNT) {
        if (vec) {
            if (lower_only) HDBF_SUB(kNT, true, true);
            else HDBF_SUB(kNT, true, false);
        } else {
            if (lower_only) HDBF_SUB(kNT, false, true);
            else HDBF_SUB(kNT, false, false);
        }
    } else if (mode == kNN) {
        if (vec) HDBF_SUB(kNN, true, false);
        else HDBF_SUB(kNN, false, false);
    } else {
        if (vec) HDBF_SUB(kTN, true, false);
        else HDBF_SUB(kTN, false, false);
    }
#undef HDBF_SUB
    ctx->launches += part ? 2 : 1;
    return last_cuda(ctx);
}

}  // namespace

hdbf_status sgemm_sub(hdbf_context* ctx, bool nn, bool lower_only, int M, int N, int K,
                      const float* A, long long lda, const float* B, long long ldb,
                      float* C, long long ldc)
{
    return sgemm_launch(ctx, nn ? kNN : kNT, lower_only, M, N, K, A, lda, B, ldb, C, ldc);
}

hdbf_status sgemm_sub_tn(hdbf_context* ctx, int M, int N, int K, const float* A, long long lda,
                         const float* B, long long ldb, float* C, long long ldc)
{
    return sgemm_launch(ctx, kTN, false, M, N, K, A, lda, B, ldb, C, ldc);
}

}  // namespace hdbf
