// FP32 -> 16-bit (BF16 / FP16) shadow copies for the tensor-core updates.
//
// The reference converts whole operands to FP16 around every GEMM call and
// back (launch_fp32_to_fp16 / launch_fp16_to_fp32, src/kernels/fp16_convert.hip,
// used by src/gemm/mixed_gemm.cpp:37-93).  Here each factor panel is rounded
// once, right after it is final, into a K-major shadow that the TMA loads of
// every later trailing update read; an optional second shadow keeps the
// rounding residual (x - hi) for the split (3-product) precision modes.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "internal.h"

namespace hdbf {
namespace {

template <typename T>
__device__ __forceinline__ T to16(float x);
template <>
__device__ __forceinline__ __nv_bfloat16 to16<__nv_bfloat16>(float x)
{
    return __float2bfloat16_rn(x);
}
template <>
__device__ __forceinline__ __half to16<__half>(float x)
{
    return __float2half_rn(x);
}
__device__ __forceinline__ float from16(__nv_bfloat16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float from16(__half x) { return __half2float(x); }

// 32 x 32 tile transpose: dst[(r) * ldd + c] = round16(s * src[c * lds + r]).
template <typename T>
__global__ void __launch_bounds__(256) transpose16_kernel(int rows, int cols,
                                                          const float* __restrict__ src,
                                                          long long lds, T* hi, T* lo,
                                                          long long ldd, float s,
                                                          const unsigned* smax)
{
    __shared__ float tile[32][33];
    if (smax) s = pow2f_exact(panel_scale_exp(*smax));
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (int j = ty; j < 32; j += 8) {
        const int r = r0 + tx, c = c0 + j;
        tile[j][tx] = (r < rows && c < cols) ? src[(long long)c * lds + r] : 0.f;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
        const int r = r0 + i, c = c0 + tx;
        if (r < rows && c < cols) {
            const float x = s * tile[tx][i];
            const T h = to16<T>(x);
            hi[(long long)r * ldd + c] = h;
            if (lo) lo[(long long)r * ldd + c] = to16<T>(x - from16(h));
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) direct16_kernel(int rows, int cols,
                                                       const float* __restrict__ src,
                                                       long long lds, T* hi, T* lo, long long ldd,
                                                       float s, const unsigned* smax)
{
    if (smax) s = pow2f_exact(panel_scale_exp(*smax));
    const int r = blockIdx.x * 256 + threadIdx.x;
    const long long c = blockIdx.y;
    if (r >= rows || c >= cols) return;
    const float x = s * src[c * lds + r];
    const T h = to16<T>(x);
    hi[c * ldd + r] = h;
    if (lo) lo[c * ldd + r] = to16<T>(x - from16(h));
}

__global__ void panel_absmax_kernel(const float* A, long long lda, int rows, int cols,
                                    unsigned* out)
{
    float v = 0.f;
    const long long total = (long long)rows * cols;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        v = fmaxf(v, fabsf(A[(i / rows) * lda + i % rows]));
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0 && v > 0.f) atomicMax(out, __float_as_uint(v));
}

}  // namespace

hdbf_status panel_absmax(hdbf_context* ctx, const float* A, long long lda, int rows, int cols,
                         unsigned* slot)
{
    cudaMemsetAsync(slot, 0, sizeof(unsigned), ctx->stream);
    if (rows <= 0 || cols <= 0) return last_cuda(ctx);
    const long long total = (long long)rows * cols;
    long long g = (total + 255) / 256;
    if (g > 4 * (long long)ctx->sm_count) g = 4 * (long long)ctx->sm_count;
    ProfScope prof(ctx, kClsConvert, 0.0, 4.0 * (double)total);
    panel_absmax_kernel<<<(unsigned)g, 256, 0, ctx->stream>>>(A, lda, rows, cols, slot);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status convert_transpose16(hdbf_context* ctx, int fmt, int rows, int cols, const float* src,
                                long long lds, void* hi, void* lo, long long ldd, float s,
                                const unsigned* smax)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    dim3 grid((rows + 31) / 32, (cols + 31) / 32);
    ProfScope prof(ctx, kClsConvert, 0.0, (double)rows * cols * (4.0 + (lo ? 4.0 : 2.0)));
    if (fmt == kFmtBF16)
        transpose16_kernel<__nv_bfloat16><<<grid, 256, 0, ctx->stream>>>(
            rows, cols, src, lds, static_cast<__nv_bfloat16*>(hi), static_cast<__nv_bfloat16*>(lo),
            ldd, s, smax);
    else
        transpose16_kernel<__half><<<grid, 256, 0, ctx->stream>>>(
            rows, cols, src, lds, static_cast<__half*>(hi), static_cast<__half*>(lo), ldd, s, smax);
    ctx->launches++;
    return last_cuda(ctx);
}

hdbf_status convert_direct16(hdbf_context* ctx, int fmt, int rows, int cols, const float* src,
                             long long lds, void* hi, void* lo, long long ldd, float s,
                             const unsigned* smax)
{
    if (rows <= 0 || cols <= 0) return HDBF_STATUS_SUCCESS;
    dim3 grid((rows + 255) / 256, cols);
    ProfScope prof(ctx, kClsConvert, 0.0, (double)rows * cols * (4.0 + (lo ? 4.0 : 2.0)));
    if (fmt == kFmtBF16)
        direct16_kernel<__nv_bfloat16><<<grid, 256, 0, ctx->stream>>>(
            rows, cols, src, lds, static_cast<__nv_bfloat16*>(hi), static_cast<__nv_bfloat16*>(lo),
            ldd, s, smax);
    else
        direct16_kernel<__half><<<grid, 256, 0, ctx->stream>>>(
            rows, cols, src, lds, static_cast<__half*>(hi), static_cast<__half*>(lo), ldd, s, smax);
    ctx->launches++;
    return last_cuda(ctx);
}

}  // namespace hdbf
