// Wavefront block triangular solve with a few right-hand sides (nrhs <= 32
// per launch), used by POTRS / GETRS.
//
// The solve is one launch per triangle.  The matrix is cut into 64-row block
// rows; CTAs take block rows in dependency order from an atomic ticket, so a
// row only ever waits on rows whose tickets were handed out earlier (to CTAs
// that are running), which rules out deadlock for any grid size.  For its
// block row i a CTA streams the off-diagonal tiles M_ij with cp.async
// (three tiles in flight, independent of the solution), and for each
// dependency j waits on a per-block flag (acquire load, bounded), folds
// M_ij x_j into its accumulator, then applies the precomputed inverse of the
// diagonal block:  x_i = op(inv_i) (b_i - sum_j M_ij x_j).  x_i is written to
// B (column-major) and to a row-major copy that consumers read with 16-byte
// loads, then published with a release store of flag i.
//
// The effective triangle M is T itself (lower forward or upper backward) or
// T^T (lower T read transposed, backward); op(inv) is inv or inv^T in the
// same orientation, so one template flag covers both.
#include "internal.h"

namespace hdbf {
namespace {

constexpr int kWT = 256;     // threads per CTA
constexpr int kB = 64;       // block-row height
constexpr int kLd = 68;      // padded shared-memory row of a 64x64 tile
constexpr int kDepth = 3;    // tiles in flight
constexpr int kSyncFlags = 32;  // sync[0] ticket, sync[1] abort, flags from here

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
__device__ __forceinline__ void cp_async16(float* smem, const float* gmem)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem, bool valid)
{
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(s), "l"(gmem),
                 "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Tile (r, k) = M(i0 + r, j0 + k) into dst: dst[k*kLd + r] (TR false, read
// T(i0 + r, j0 + k)) or dst[r*kLd + k] (TR true, read T(j0 + k, i0 + r)).
// In both cases the contiguous global index u lands contiguously in smem.
// Entries outside the n x n matrix are zero-filled.
template <bool TR>
__device__ __forceinline__ void load_tile(float* dst, const float* T, long long ldt, int n, int i0,
                                          int j0, bool vec)
{
    const int a0 = TR ? j0 : i0, b0 = TR ? i0 : j0;
    if (vec && a0 + kB <= n && b0 + kB <= n) {
        for (int q = threadIdx.x; q < kB * kB / 4; q += kWT) {
            const int v = q >> 4, u = (q & 15) * 4;
            cp_async16(dst + v * kLd + u, T + (a0 + u) + (long long)(b0 + v) * ldt);
        }
    } else {
        for (int q = threadIdx.x; q < kB * kB; q += kWT) {
            const int v = q >> 6, u = q & 63;
            const bool ok = a0 + u < n && b0 + v < n;
            cp_async4(dst + v * kLd + u, ok ? T + (a0 + u) + (long long)(b0 + v) * ldt : T, ok);
        }
    }
}

template <int NB, bool TR>
__global__ void __launch_bounds__(kWT, 2) trsv_wave_kernel(int n, int nrhs, const float* __restrict__ T,
                                                        long long ldt, int vec,
                                                        const float* __restrict__ inv, int backward,
                                                        float* B, long long ldb, float* X,
                                                        int* sync, int* err)
{
    constexpr int XS = NB + 4;    // padded row of the x / y staging tiles
    constexpr int CW = NB / 4;    // columns per thread in the diagonal step
    extern __shared__ __align__(16) float smem[];
    float* Mt = smem;                          // kDepth tiles
    float* Is = Mt + kDepth * kB * kLd;        // op(inv_i)
    float* Xs = Is + kB * kLd;                 // x_j (row-major, padded); later y_i
    float* red = Mt;                           // 4 x NB x 64 partial sums (after the tiles)
    __shared__ int s_ticket, s_abort;

    const int tid = threadIdx.x;
    const int nb = (n + kB - 1) / kB;
    unsigned* flags = reinterpret_cast<unsigned*>(sync + kSyncFlags);
    int* abortp = sync + 1;
    const int r = tid & 63, g = tid >> 6;

    if (tid == 0) s_abort = 0;
    for (;;) {
        if (tid == 0) s_ticket = atomicAdd(sync, 1);
        __syncthreads();
        const int p = s_ticket;
        if (p >= nb) return;
        const int i = backward ? nb - 1 - p : p;
        const int i0 = i * kB;
        const int rows = min(kB, n - i0);
        const int m = backward ? nb - 1 - i : i;  // number of dependencies

        // prologue: inverse block, first kDepth tiles, right-hand side
        {
            const float* src = inv + (long long)i * kB * kB;
            for (int q = tid; q < kB * kB / 4; q += kWT) {
                const int v = q >> 4, u = (q & 15) * 4;
                cp_async16(Is + v * kLd + u, src + v * kB + u);
            }
            cp_commit();
        }
#pragma unroll
        for (int d = 0; d < kDepth; ++d) {
            if (d < m) {
                const int j = backward ? nb - 1 - d : d;
                load_tile<TR>(Mt + d * kB * kLd, T, ldt, n, i0, j * kB, vec != 0);
            }
            cp_commit();
        }
        float bv[CW];
#pragma unroll
        for (int c = 0; c < CW; ++c) {
            const int col = g * CW + c;
            bv[c] = (r < rows && col < nrhs) ? B[(long long)col * ldb + i0 + r] : 0.f;
        }
        float acc[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) acc[c] = 0.f;

        for (int s = 0; s < m; ++s) {
            const int j = backward ? nb - 1 - s : s;
            if (tid == 0) {
                unsigned polls = 0;
                while (ld_acquire_u32(flags + j) == 0u) {
                    if (*reinterpret_cast<volatile int*>(abortp)) { s_abort = 1; break; }
                    if (++polls > spin_limit_of(err)) {
                        atomicCAS(err, 0, kErrTimeout);
                        atomicExch(abortp, 1);
                        s_abort = 1;
                        break;
                    }
                    if (polls > 32) __nanosleep(64);
                }
            }
            cp_wait<kDepth - 1>();
            __syncthreads();
            if (s_abort) {
                cp_wait<0>();
                return;
            }
            {
                const float4* xsrc = reinterpret_cast<const float4*>(X + (long long)j * kB * NB);
                for (int q = tid; q < kB * NB / 4; q += kWT) {
                    const int k = q / (NB / 4), c4 = q - k * (NB / 4);
                    *reinterpret_cast<float4*>(Xs + k * XS + 4 * c4) = __ldcg(xsrc + q);
                }
            }
            __syncthreads();
            const float* S = Mt + (s % kDepth) * kB * kLd;
#pragma unroll
            for (int kq = 0; kq < 4; ++kq) {
                const int kb = g * 16 + kq * 4;
                float a[4];
                if (TR) {
                    const float4 v = *reinterpret_cast<const float4*>(S + r * kLd + kb);
                    a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) a[e] = S[(kb + e) * kLd + r];
                }
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float4* xr = reinterpret_cast<const float4*>(Xs + (kb + e) * XS);
#pragma unroll
                    for (int q = 0; q < NB / 4; ++q) {
                        const float4 xv = xr[q];
                        acc[4 * q + 0] = fmaf(a[e], xv.x, acc[4 * q + 0]);
                        acc[4 * q + 1] = fmaf(a[e], xv.y, acc[4 * q + 1]);
                        acc[4 * q + 2] = fmaf(a[e], xv.z, acc[4 * q + 2]);
                        acc[4 * q + 3] = fmaf(a[e], xv.w, acc[4 * q + 3]);
                    }
                }
            }
            __syncthreads();
            if (s + kDepth < m) {
                const int jn = backward ? nb - 1 - (s + kDepth) : s + kDepth;
                load_tile<TR>(Mt + (s % kDepth) * kB * kLd, T, ldt, n, i0, jn * kB, vec != 0);
            }
            cp_commit();
        }
        cp_wait<0>();
        __syncthreads();

        // y_i = b_i - sum over the four k-groups
#pragma unroll
        for (int c = 0; c < NB; ++c) red[(g * NB + c) * kB + r] = acc[c];
        __syncthreads();
#pragma unroll
        for (int c = 0; c < CW; ++c) {
            const int col = g * CW + c;
            float y = bv[c];
#pragma unroll
            for (int q = 0; q < 4; ++q) y -= red[(q * NB + col) * kB + r];
            Xs[r * XS + col] = (r < rows) ? y : 0.f;
        }
        __syncthreads();

        // x_i = op(inv_i) y_i
        float x[CW];
#pragma unroll
        for (int c = 0; c < CW; ++c) x[c] = 0.f;
#pragma unroll 4
        for (int k = 0; k < kB; k += 4) {
            float a[4];
            if (TR) {
                const float4 v = *reinterpret_cast<const float4*>(Is + r * kLd + k);
                a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) a[e] = Is[(k + e) * kLd + r];
            }
#pragma unroll
            for (int e = 0; e < 4; ++e)
#pragma unroll
                for (int c = 0; c < CW; ++c) x[c] = fmaf(a[e], Xs[(k + e) * XS + g * CW + c], x[c]);
        }
        float* xdst = X + (long long)(i0 + r) * NB + g * CW;
#pragma unroll
        for (int c = 0; c < CW; ++c) {
            const int col = g * CW + c;
            const bool ok = r < rows && col < nrhs;
            if (ok) B[(long long)col * ldb + i0 + r] = x[c];
            xdst[c] = ok ? x[c] : 0.f;
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release_u32(flags + i, 1u);
        }
    }
}

template <int NB, bool TR>
size_t wave_smem() { return sizeof(float) * ((kDepth + 1) * kB * kLd + kB * (NB + 4)); }

template <int NB, bool TR>
hdbf_status wave_launch(hdbf_context* ctx, int n, int nc, const float* T, long long ldt, int vec,
                        const float* inv, int backward, float* B, long long ldb, float* X,
                        int* sync)
{
    const size_t smem = wave_smem<NB, TR>();
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsv_wave_kernel<NB, TR>, kWT, smem);
    if (per_sm < 1) per_sm = 1;
    const int nb = (n + kB - 1) / kB;
    const int grid = nb < per_sm * ctx->sm_count ? nb : per_sm * ctx->sm_count;
    trsv_wave_kernel<NB, TR><<<grid, kWT, smem, ctx->stream>>>(
        n, nc, T, ldt, vec, inv, backward, B, ldb, X, sync, ctx->dev_small + kSmallErr);
    ctx->launches++;
    return last_cuda(ctx);
}

template <int NB, bool TR>
void wave_configure()
{
    cudaFuncSetAttribute(trsv_wave_kernel<NB, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)wave_smem<NB, TR>());
}

}  // namespace

size_t wave_scratch_bytes(int n)
{
    const size_t nb = (size_t)((n < 1 ? 1 : n) + kB - 1) / kB;
    return align_up(nb * kB * 32 * sizeof(float), 256) +
           align_up((nb + kSyncFlags) * sizeof(int), 256);
}

void configure_wave_kernels(hdbf_context*)
{
    wave_configure<8, false>();
    wave_configure<16, false>();
    wave_configure<32, false>();
    wave_configure<8, true>();
    wave_configure<16, true>();
    wave_configure<32, true>();
    cudaGetLastError();
}

hdbf_status trsv_wave(hdbf_context* ctx, int n, int nrhs, const float* T, long long ldt, bool trans,
                      const float* inv, bool backward, float* B, long long ldb)
{
    if (n <= 0 || nrhs <= 0) return HDBF_STATUS_SUCCESS;
    if (!T || !inv || !B || ldt < n || ldb < n) return HDBF_STATUS_INVALID_VALUE;
    HDBF_TRY(ensure_ws(ctx, n));
    const int nb = (n + kB - 1) / kB;
    float* X = ws_wave(ctx);
    int* sync = reinterpret_cast<int*>(
        reinterpret_cast<char*>(X) + align_up((size_t)nb * kB * 32 * sizeof(float), 256));
    const int vec = ((reinterpret_cast<uintptr_t>(T) & 15) == 0 && ldt % 4 == 0) ? 1 : 0;
    for (int c0 = 0; c0 < nrhs; c0 += 32) {
        const int nc = nrhs - c0 < 32 ? nrhs - c0 : 32;
        float* Bc = B + (long long)c0 * ldb;
        if (cudaMemsetAsync(sync, 0, (size_t)(nb + kSyncFlags) * sizeof(int), ctx->stream) !=
            cudaSuccess)
            return last_cuda(ctx);
        ProfScope prof(ctx, kClsWave, (double)n * n * nc,
                       2.0 * (double)n * n + 8.0 * (double)n * nc, n, nc, n);
        hdbf_status st;
        if (nc <= 8)
            st = trans ? wave_launch<8, true>(ctx, n, nc, T, ldt, vec, inv, backward, Bc, ldb, X, sync)
                       : wave_launch<8, false>(ctx, n, nc, T, ldt, vec, inv, backward, Bc, ldb, X, sync);
        else if (nc <= 16)
            st = trans ? wave_launch<16, true>(ctx, n, nc, T, ldt, vec, inv, backward, Bc, ldb, X, sync)
                       : wave_launch<16, false>(ctx, n, nc, T, ldt, vec, inv, backward, Bc, ldb, X, sync);
        else
            st = trans ? wave_launch<32, true>(ctx, n, nc, T, ldt, vec, inv, backward, Bc, ldb, X, sync)
                       : wave_launch<32, false>(ctx, n, nc, T, ldt, vec, inv, backward, Bc, ldb, X, sync);
        if (st != HDBF_STATUS_SUCCESS) return st;
    }
    return HDBF_STATUS_SUCCESS;
}

}  // namespace hdbf
