// Mixed-precision trailing update on the 5th-generation tensor cores:
//     C (FP32, column-major, in place) -= scale * A * B^T
// with A (M x K) and B (N x K) stored K-major in 16-bit (BF16 or FP16)
// "shadow" copies, products accumulated in FP32 in tensor memory.
//
// Replaces the reference's FP16 GEMM path (launch_mixed_gemm,
// src/gemm/mixed_gemm.cpp:8-96: rocblas_gemm_ex with FP16 inputs AND an FP16
// C), here with an FP32 C: every trailing update is applied to the FP32
// master matrix, only the two input operands are rounded to 16 bits.
//
// Kernel: one 128 x 128 output tile per CTA (4 warps), two CTAs per SM.  Warp 0 / lane 0 feeds
// a STAGES-deep shared-memory ring with TMA tile loads (128 rows x 64
// elements of A and of B per stage, 128-byte swizzle, no multicast); warp 1 /
// lane 0 issues tcgen05.mma (kind::f16, M=128, N=128, K=16) into a 128-column
// TMEM accumulator and frees ring slots with tcgen05.commit; after the last
// MMA all four warps read the accumulator back with tcgen05.ld (each warp its
// own 32-lane TMEM sub-partition) and update C with coalesced FP32
// read-modify-writes.  Every mbarrier wait is bounded: on expiry the kernel
// records an error, drains what it issued, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "internal.h"

namespace hdbf {
namespace {

constexpr int TM = 128;
constexpr int TN = 128;
constexpr int TK = 64;  // 64 x 16-bit = 128 bytes = one swizzle row
constexpr int A_BYTES = TM * TK * 2;
constexpr int B_BYTES = TN * TK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int TMEM_COLS = 128;
// One product: 3 stages of (A, B), 2 CTAs per SM (one's epilogue overlaps the
// other's main loop).  Split (hi/lo) operands: 2 stages of (A, B, A_lo, B_lo)
// and the three products hi*hi + hi*lo + lo*hi into one accumulator, 1 CTA/SM.
template <bool SPLIT>
struct TcCfg {
    static constexpr int kStages = SPLIT ? 2 : 3;
    static constexpr int kStageBytes = SPLIT ? 2 * STAGE_BYTES : STAGE_BYTES;
    static constexpr size_t kSmem = (size_t)kStages * kStageBytes + 1024;  // + alignment slack
};
constexpr long long kWaitCycles = 4000000000LL;                   // ~2 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase; false (and *err set) on expiry.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > kWaitCycles) {
            atomicCAS(err, 0, kErrTimeout);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), LBO unused for swizzled K-major, version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor, kind::f16: FP32 accumulate, A/B = BF16 (fmt 1) or
// FP16 (fmt 0), both K-major, N = 128, M = 128.
__host__ __device__ constexpr uint32_t make_idesc(int fmt)
{
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(TN >> 3) << 17) |
           ((uint32_t)(TM >> 4) << 24);
}

struct TcArgs {
    int M, N, K;
    int a_row0, a_k0, b_row0, b_k0;
    float* C;
    long long ldc;
    float scale;
    const unsigned* sa_max;  // optional per-panel scale sources (panel_scale_exp)
    const unsigned* sb_max;
    int tiles_m;
    int lower;
    int fmt;
    int* err;
};

template <bool SPLIT>
__global__ void __launch_bounds__(128, SPLIT ? 1 : 2)
tc_gemm_sub_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                   const __grid_constant__ CUtensorMap mapAl,
                   const __grid_constant__ CUtensorMap mapBl, const TcArgs args)
{
    constexpr int STAGES = TcCfg<SPLIT>::kStages;
    constexpr int SB = TcCfg<SPLIT>::kStageBytes;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    __shared__ __align__(8) uint64_t empty_bar[STAGES];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;

    const int tm = blockIdx.x % args.tiles_m;
    const int tn = blockIdx.x / args.tiles_m;
    const int m0 = tm * TM, n0 = tn * TN;
    if (args.lower && m0 + TM <= n0) return;  // tile strictly above the diagonal

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                               ~static_cast<uintptr_t>(1023));
    // stage s: [A | B | A_lo | B_lo] (each tile 1024-byte aligned)
    auto sA = [&](int st) { return smem + st * SB; };
    auto sB = [&](int st) { return smem + st * SB + A_BYTES; };
    auto sAl = [&](int st) { return smem + st * SB + STAGE_BYTES; };
    auto sBl = [&](int st) { return smem + st * SB + STAGE_BYTES + A_BYTES; };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&done_bar, 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t taddr = tmem_slot;
    const int ktiles = (args.K + TK - 1) / TK;

    if (warp == 0 && lane == 0) {
        // TMA producer
        for (int kt = 0; kt < ktiles; ++kt) {
            const int s = kt % STAGES;
            if (kt >= STAGES && !mbar_wait(&empty_bar[s], ((kt / STAGES) - 1) & 1, args.err)) {
                s_fail = 1;
                break;
            }
            mbar_expect_tx(&full_bar[s], SB);
            tma_load_2d(sA(s), &mapA, &full_bar[s], args.a_k0 + kt * TK, args.a_row0 + m0);
            tma_load_2d(sB(s), &mapB, &full_bar[s], args.b_k0 + kt * TK, args.b_row0 + n0);
            if (SPLIT) {
                tma_load_2d(sAl(s), &mapAl, &full_bar[s], args.a_k0 + kt * TK, args.a_row0 + m0);
                tma_load_2d(sBl(s), &mapBl, &full_bar[s], args.b_k0 + kt * TK, args.b_row0 + n0);
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        const uint32_t idesc = make_idesc(args.fmt);
        for (int kt = 0; kt < ktiles; ++kt) {
            const int s = kt % STAGES;
            if (!mbar_wait(&full_bar[s], (kt / STAGES) & 1, args.err)) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sA(s));
            const uint32_t b0 = smem_u32(sB(s));
            const uint32_t al0 = smem_u32(sAl(s));
            const uint32_t bl0 = smem_u32(sBl(s));
            auto mma = [&](uint64_t ad, uint64_t bd, uint32_t acc) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
            };
#pragma unroll
            for (int kk = 0; kk < TK / 16; ++kk) {
                const uint64_t ad = sw128_desc(a0 + kk * 32);
                const uint64_t bd = sw128_desc(b0 + kk * 32);
                mma(ad, bd, (kt > 0 || kk > 0) ? 1u : 0u);
                if (SPLIT) {
                    mma(ad, sw128_desc(bl0 + kk * 32), 1u);
                    mma(sw128_desc(al0 + kk * 32), bd, 1u);
                }
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&empty_bar[s]))
                : "memory");
        }
        // done_bar fires once every MMA issued above has completed.
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(&done_bar))
            : "memory");
    }

    // Prefetch this thread's first 32 C values while the MMAs drain.
    const int row = m0 + warp * 32 + lane;
    float cv[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const int col = n0 + j;
        cv[j] = (row < args.M && col < args.N) ? __ldcg(args.C + (long long)col * args.ldc + row)
                                               : 0.f;
    }
    __syncwarp();
    const bool ok = mbar_wait(&done_bar, 0, args.err);
    asm volatile("tcgen05.fence::after_thread_sync;");
    __syncthreads();
    if (ok && !s_fail && ktiles > 0) {
        float scale = args.scale;  // undo the operands' per-panel scales
        if (args.sa_max) scale *= pow2f_exact(-panel_scale_exp(*args.sa_max));
        if (args.sb_max) scale *= pow2f_exact(-panel_scale_exp(*args.sb_max));
        const uint32_t lane_base = taddr + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < TN; c0 += 32) {
            if (c0 > 0) {  // all 32 loads of the chunk in flight together
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + c0 + j;
                    cv[j] = (row < args.M && col < args.N)
                                ? __ldcg(args.C + (long long)col * args.ldc + row)
                                : 0.f;
                }
            }
            uint32_t v[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                  "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                  "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                  "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                  "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                  "=r"(v[30]), "=r"(v[31])
                : "r"(lane_base + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < args.M) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < args.N && (!args.lower || row >= col))
                        args.C[(long long)col * args.ldc + row] =
                            fmaf(-scale, __uint_as_float(v[j]), cv[j]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                     "r"(TMEM_COLS));
}

// ------------------------------------------------ persistent 128 x 256 kernel
// One CTA per SM walks the output tiles (128 x 256, band by band of 256
// columns; with `lower` only the tiles that reach the diagonal or below) in
// a fixed stride of the grid size.  Warp roles:
//   warp 0 / lane 0   TMA producer: A (128 x 64) and B (256 x 64) per stage
//                     into a STAGES-deep ring, continuing across tiles;
//   warp 1 / lane 0   MMA issuer: tcgen05.mma M=128, N=256, K=16 into one of
//                     two 256-column TMEM accumulators (tile i uses i & 1),
//                     so the next tile's products run while the epilogue
//                     drains the previous one;
//   warps 2..5        epilogue: tcgen05.ld of their 32-lane sub-partition in
//                     32-column chunks, C -= scale * acc with coalesced FP32
//                     read-modify-writes, then release the accumulator.
// Barriers: full/empty per ring stage, tmem_full/tmem_empty per accumulator.
// Every wait is bounded; on expiry (or when another role gave up) the role
// records kErrTimeout, stops, and the CTA drains its MMAs before freeing TMEM.
constexpr int PN = 256;
constexpr int PB_BYTES = PN * TK * 2;
constexpr int P_STAGE = A_BYTES + PB_BYTES;
constexpr int P_TMEM_COLS = 2 * PN;
constexpr int kPThreads = 192;
template <bool SPLIT>
struct PCfg {
    static constexpr int kStages = SPLIT ? 2 : 4;
    static constexpr int kStageBytes = SPLIT ? 2 * P_STAGE : P_STAGE;
    static constexpr size_t kSmem = (size_t)kStages * kStageBytes + 1024;
};

__host__ __device__ constexpr uint32_t make_idesc_n(int fmt, int n)
{
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(TM >> 4) << 24);
}

// Bounded wait that also gives up once another role of the CTA has failed.
__device__ __forceinline__ bool mbar_wait_or_fail(uint64_t* bar, uint32_t parity, int* err,
                                                  volatile int* fail)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (*fail) return false;
        if (clock64() - t0 > kWaitCycles) {
            atomicCAS(err, 0, kErrTimeout);
            *fail = 1;
            return false;
        }
    }
    return true;
}

struct PArgs {
    int M, N, K;
    int a_row0, a_k0, b_row0, b_k0;
    float* C;
    long long ldc;
    float scale;
    const unsigned* sa_max;
    const unsigned* sb_max;
    int tiles_m, tiles_n;
    long long total;  // tiles to compute
    int lower;
    int fmt;
    int* err;
};

// Linear tile index -> (tm, tn), band by band (tn outer); the cursor only
// moves forward, as every role visits its tiles in increasing order.
struct TileWalk {
    int tn = 0;
    long long base = 0;
    __device__ __forceinline__ void locate(const PArgs& a, long long t, int& tm, int& tnn)
    {
        for (;;) {
            const long long cnt = a.lower ? (long long)max(0, a.tiles_m - 2 * tn) : a.tiles_m;
            if (t < base + cnt || tn >= a.tiles_n - 1) {
                tm = (a.lower ? 2 * tn : 0) + (int)(t - base);
                tnn = tn;
                return;
            }
            base += cnt;
            ++tn;
        }
    }
};

template <bool SPLIT>
__global__ void __launch_bounds__(kPThreads, 1)
tc_gemm_persistent_kernel(const __grid_constant__ CUtensorMap mapA,
                          const __grid_constant__ CUtensorMap mapB,
                          const __grid_constant__ CUtensorMap mapAl,
                          const __grid_constant__ CUtensorMap mapBl, const PArgs args)
{
    constexpr int STAGES = PCfg<SPLIT>::kStages;
    constexpr int SB = PCfg<SPLIT>::kStageBytes;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    __shared__ __align__(8) uint64_t empty_bar[STAGES];
    __shared__ __align__(8) uint64_t tfull_bar[2];
    __shared__ __align__(8) uint64_t tempty_bar[2];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_slot;
    __shared__ int s_fail;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                               ~static_cast<uintptr_t>(1023));
    // stage s: [A | B | A_lo | B_lo] (each tile 1024-byte aligned)
    auto sA = [&](int st) { return smem + st * SB; };
    auto sB = [&](int st) { return smem + st * SB + A_BYTES; };
    auto sAl = [&](int st) { return smem + st * SB + P_STAGE; };
    auto sBl = [&](int st) { return smem + st * SB + P_STAGE + A_BYTES; };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int* fail = &s_fail;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(P_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull_bar[b], 1);
            mbar_init(&tempty_bar[b], 4);  // one arrival per epilogue warp
        }
        mbar_init(&done_bar, 1);
        s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t taddr = tmem_slot;
    const int ktiles = (args.K + TK - 1) / TK;
    const long long G = gridDim.x;


    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            TileWalk walk;
            uint32_t it = 0;
            bool ok = true;
            for (long long t = blockIdx.x; t < args.total && ok; t += G) {
                int tm, tn;
                walk.locate(args, t, tm, tn);
                const int m0 = tm * TM, n0 = tn * PN;
                for (int kt = 0; kt < ktiles; ++kt, ++it) {
                    const int s = (int)(it % STAGES);
                    if (it >= (uint32_t)STAGES &&
                        !mbar_wait_or_fail(&empty_bar[s], ((it / STAGES) - 1) & 1, args.err, fail)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full_bar[s], SB);
                    const int kx = args.a_k0 + kt * TK, kb = args.b_k0 + kt * TK;
                    tma_load_2d(sA(s), &mapA, &full_bar[s], kx, args.a_row0 + m0);
                    tma_load_2d(sB(s), &mapB, &full_bar[s], kb, args.b_row0 + n0);
                    if (SPLIT) {
                        tma_load_2d(sAl(s), &mapAl, &full_bar[s], kx, args.a_row0 + m0);
                        tma_load_2d(sBl(s), &mapBl, &full_bar[s], kb, args.b_row0 + n0);
                    }
                }
            }
            if (!ok) {  // let the copies already issued land before the CTA exits
                const uint32_t first = it > (uint32_t)STAGES ? it - STAGES : 0u;
                for (uint32_t q = first; q < it; ++q) {
                    const long long t0 = clock64();
                    while (!mbar_try_wait(&full_bar[q % STAGES], (q / STAGES) & 1) &&
                           clock64() - t0 < kWaitCycles) {
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            const uint32_t idesc = make_idesc_n(args.fmt, PN);
            uint32_t it = 0;
            int local = 0;
            bool ok = true;
            for (long long t = blockIdx.x; t < args.total && ok; t += G, ++local) {
                const int buf = local & 1;
                if (local >= 2 &&
                    !mbar_wait_or_fail(&tempty_bar[buf], ((local >> 1) - 1) & 1, args.err, fail)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t d = taddr + (uint32_t)(buf * PN);
                for (int kt = 0; kt < ktiles; ++kt, ++it) {
                    const int s = (int)(it % STAGES);
                    if (!mbar_wait_or_fail(&full_bar[s], (it / STAGES) & 1, args.err, fail)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t a0 = smem_u32(sA(s)), b0 = smem_u32(sB(s));
                    const uint32_t al0 = smem_u32(sAl(s)), bl0 = smem_u32(sBl(s));
                    auto mma = [&](uint64_t ad, uint64_t bd, uint32_t acc) {
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
                            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
                    };
#pragma unroll
                    for (int kk = 0; kk < TK / 16; ++kk) {
                        const uint64_t ad = sw128_desc(a0 + kk * 32);
                        const uint64_t bd = sw128_desc(b0 + kk * 32);
                        mma(ad, bd, (kt > 0 || kk > 0) ? 1u : 0u);
                        if (SPLIT) {
                            mma(ad, sw128_desc(bl0 + kk * 32), 1u);
                            mma(sw128_desc(al0 + kk * 32), bd, 1u);
                        }
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                        "[%0];" ::"r"(smem_u32(&empty_bar[s]))
                        : "memory");
                }
                if (!ok) break;
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                        smem_u32(&tfull_bar[buf]))
                    : "memory");
            }
            // done_bar fires once every MMA issued above has completed.
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&done_bar))
                : "memory");
            const long long t0 = clock64();
            while (!mbar_try_wait(&done_bar, 0) && clock64() - t0 < kWaitCycles) {
            }
        }
    } else {  // epilogue: warps 2..5, TMEM sub-partition warp % 4
        const int sub = warp & 3;
        float scale = args.scale;  // undo the operands' per-panel scales
        if (args.sa_max) scale *= pow2f_exact(-panel_scale_exp(*args.sa_max));
        if (args.sb_max) scale *= pow2f_exact(-panel_scale_exp(*args.sb_max));
        TileWalk walk;
        int local = 0;
        for (long long t = blockIdx.x; t < args.total; t += G, ++local) {
            int tm, tn;
            walk.locate(args, t, tm, tn);
            const int m0 = tm * TM, n0 = tn * PN;
            const int buf = local & 1;
            const int row = m0 + sub * 32 + lane;
            const bool row_ok = row < args.M;
            float cv[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {  // first chunk of C while the MMAs run
                const int col = n0 + j;
                cv[j] = (row_ok && col < args.N) ? __ldcg(args.C + (long long)col * args.ldc + row)
                                                 : 0.f;
            }
            // warp-uniform outcome: tcgen05.ld below needs the whole warp
            const bool ready = mbar_wait_or_fail(&tfull_bar[buf], (local >> 1) & 1, args.err, fail);
            if (!__all_sync(0xffffffffu, ready)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t lane_base = taddr + ((uint32_t)(sub * 32) << 16) + (uint32_t)(buf * PN);
#pragma unroll 1
            for (int c0 = 0; c0 < PN; c0 += 32) {
                uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                      "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                      "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
                      "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]),
                      "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(lane_base + (uint32_t)c0));
            float nx[32];  // next chunk of C, in flight during this chunk's stores
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int col = n0 + c0 + 32 + j;
                nx[j] = (c0 + 32 < PN && row_ok && col < args.N)
                            ? __ldcg(args.C + (long long)col * args.ldc + row)
                            : 0.f;
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (c0 + 32 >= PN) {  // accumulator read out: hand it back to the MMA warp
                asm volatile("tcgen05.fence::before_thread_sync;");
                __syncwarp();
                if (lane == 0)
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                                     smem_u32(&tempty_bar[buf]))
                                 : "memory");
            }
            if (row_ok) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < args.N && (!args.lower || row >= col))
                        args.C[(long long)col * args.ldc + row] =
                            fmaf(-scale, __uint_as_float(v[j]), cv[j]);
                }
            }
#pragma unroll
                for (int j = 0; j < 32; ++j) cv[j] = nx[j];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr),
                     "r"(P_TMEM_COLS));
}

// --------------------------------------------------------------- tensor maps
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

// 2-D map over a K-major 16-bit matrix: dims (k_extent, row_extent), row
// stride ld elements; box 64 x box_rows with 128-byte swizzle; reads outside
// the extents return zero.
bool make_map(CUtensorMap* map, const void* base, long long ld, long long row_extent,
              long long k_extent, int fmt, int box_rows = TM)
{
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)k_extent, (cuuint64_t)row_extent};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)TK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUtensorMapDataType dt =
        fmt == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const CUresult r = fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

void configure_tc_kernels(hdbf_context* ctx)
{
    (void)ctx;
    cudaFuncSetAttribute(tc_gemm_sub_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TcCfg<false>::kSmem);
    cudaFuncSetAttribute(tc_gemm_sub_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TcCfg<true>::kSmem);
    cudaFuncSetAttribute(tc_gemm_persistent_kernel<false>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PCfg<false>::kSmem);
    cudaFuncSetAttribute(tc_gemm_persistent_kernel<true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PCfg<true>::kSmem);
    cudaGetLastError();
}

namespace {
hdbf_status tc_launch(hdbf_context* ctx, int fmt, int M, int N, int K, const TcOperand& A,
                      const TcOperand& B, const TcOperand* Alo, const TcOperand* Blo, float* C,
                      long long ldc, float scale, bool lower_only, const unsigned* sa_max,
                      const unsigned* sb_max)
{
    if (M <= 0 || N <= 0 || K <= 0) return HDBF_STATUS_SUCCESS;
    const bool split = Alo && Blo;
    const TcOperand* ops[4] = {&A, &B, Alo, Blo};
    for (int q = 0; q < (split ? 4 : 2); ++q) {
        const TcOperand& o = *ops[q];
        // TMA: 16-byte aligned base and row stride; the K coordinate of every
        // tile must start on a 16-byte (8-element) boundary.
        if (!o.base || (reinterpret_cast<uintptr_t>(o.base) & 15u) || (o.ld % 8) || (o.k0 % 8))
            return HDBF_STATUS_INVALID_VALUE;
    }
    if (!C) return HDBF_STATUS_INVALID_VALUE;
    if (split && (Alo->row0 != A.row0 || Alo->k0 != A.k0 || Blo->row0 != B.row0 || Blo->k0 != B.k0))
        return HDBF_STATUS_INVALID_VALUE;
    const bool persistent = ctx->tc_kernel == 0;
    const int brows = persistent ? PN : TN;  // B tile rows per TMA box
    CUtensorMap ma, mb, mal, mbl;
    if (!make_map(&ma, A.base, A.ld, (long long)A.row0 + M, (long long)A.k0 + K, fmt) ||
        !make_map(&mb, B.base, B.ld, (long long)B.row0 + N, (long long)B.k0 + K, fmt, brows))
        return HDBF_STATUS_NOT_SUPPORTED;
    if (split) {
        if (!make_map(&mal, Alo->base, Alo->ld, (long long)A.row0 + M, (long long)A.k0 + K, fmt) ||
            !make_map(&mbl, Blo->base, Blo->ld, (long long)B.row0 + N, (long long)B.k0 + K, fmt,
                      brows))
            return HDBF_STATUS_NOT_SUPPORTED;
    } else {
        mal = ma;
        mbl = mb;
    }
    TcArgs args;
    args.M = M;
    args.N = N;
    args.K = K;
    args.a_row0 = A.row0;
    args.a_k0 = A.k0;
    args.b_row0 = B.row0;
    args.b_k0 = B.k0;
    args.C = C;
    args.ldc = ldc;
    args.scale = scale;
    args.sa_max = sa_max;
    args.sb_max = sb_max;
    args.tiles_m = (M + TM - 1) / TM;
    args.lower = lower_only ? 1 : 0;
    args.fmt = fmt;
    args.err = ctx->dev_small + kSmallErr;
    const long long grid = (long long)args.tiles_m * ((N + TN - 1) / TN);
    if (grid > 0x7fffffffLL) return HDBF_STATUS_NOT_SUPPORTED;
    // Algorithmic flops: with lower_only only the entries row >= col of C are
    // updated (the kernel skips tiles above the diagonal), so count
    // sum over columns j < min(M, N) of (M - j) rows, as the FP32 GEMM does.
    double entries = (double)M * N;
    if (lower_only) {
        const double d = (double)(M < N ? M : N);
        entries = d * (double)M - d * (d - 1.0) / 2.0;
    }
    const double flops = (split ? 3.0 : 1.0) * 2.0 * entries * K;
    ProfScope prof(ctx, kClsTcGemm, flops,
                   (split ? 4.0 : 2.0) * ((double)M * K + (double)N * K) + 8.0 * M * N, M, N, K);
    if (persistent) {
        PArgs pa;
        pa.M = M;
        pa.N = N;
        pa.K = K;
        pa.a_row0 = A.row0;
        pa.a_k0 = A.k0;
        pa.b_row0 = B.row0;
        pa.b_k0 = B.k0;
        pa.C = C;
        pa.ldc = ldc;
        pa.scale = scale;
        pa.sa_max = sa_max;
        pa.sb_max = sb_max;
        pa.tiles_m = args.tiles_m;
        pa.tiles_n = (N + PN - 1) / PN;
        pa.lower = args.lower;
        pa.fmt = fmt;
        pa.err = args.err;
        long long total = 0;  // tiles reaching the diagonal or below (lower), else all
        for (int tn = 0; tn < pa.tiles_n; ++tn)
            total += lower_only ? std::max(0, pa.tiles_m - 2 * tn) : pa.tiles_m;
        pa.total = total;
        if (total <= 0) return HDBF_STATUS_SUCCESS;
        const unsigned g = (unsigned)std::min<long long>(total, ctx->sm_count);
        if (split)
            tc_gemm_persistent_kernel<true><<<g, kPThreads, PCfg<true>::kSmem, ctx->stream>>>(
                ma, mb, mal, mbl, pa);
        else
            tc_gemm_persistent_kernel<false><<<g, kPThreads, PCfg<false>::kSmem, ctx->stream>>>(
                ma, mb, mal, mbl, pa);
    } else if (split) {
        tc_gemm_sub_kernel<true><<<(unsigned)grid, 128, TcCfg<true>::kSmem, ctx->stream>>>(
            ma, mb, mal, mbl, args);
    } else {
        tc_gemm_sub_kernel<false><<<(unsigned)grid, 128, TcCfg<false>::kSmem, ctx->stream>>>(
            ma, mb, mal, mbl, args);
    }
    ctx->launches++;
    return last_cuda(ctx);
}
}  // namespace

hdbf_status tc_gemm_sub(hdbf_context* ctx, int fmt, int M, int N, int K, const TcOperand& A,
                        const TcOperand& B, float* C, long long ldc, float scale, bool lower_only,
                        const unsigned* sa_max, const unsigned* sb_max)
{
    return tc_launch(ctx, fmt, M, N, K, A, B, nullptr, nullptr, C, ldc, scale, lower_only, sa_max,
                     sb_max);
}

hdbf_status tc_gemm_sub_split(hdbf_context* ctx, int fmt, int M, int N, int K, const TcOperand& A,
                              const TcOperand& Alo, const TcOperand& B, const TcOperand& Blo,
                              float* C, long long ldc, float scale, bool lower_only,
                              const unsigned* sa_max, const unsigned* sb_max)
{
    return tc_launch(ctx, fmt, M, N, K, A, B, &Alo, &Blo, C, ldc, scale, lower_only, sa_max,
                     sb_max);
}

}  // namespace hdbf
