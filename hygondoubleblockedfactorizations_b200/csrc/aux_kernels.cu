// Auxiliary device kernels: damping, FP32<->FP16 copies, SPD auto-scaling,
// the counter-based input generator and pivot offsetting.
//
// Reference counterparts: src/kernels/add_damping.hip:10-66,
// src/kernels/fp16_convert.hip:12-129, src/kernels/matrix_scale.hip:10-113.
#include <cuda_fp16.h>

#include "internal.h"
#include "kernels/add_damping.h"
#include "kernels/fp16_convert.h"
#include "kernels/matrix_scale.h"

namespace hdbf {
namespace {

template <typename T>
__global__ void add_damping_kernel(T* A, int n, long long lda, T lambda)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) A[(long long)i * lda + i] += lambda;
}

// Column-major copy with leading-dimension change; grid (row blocks, cols).
__global__ void f32_to_f16_kernel(const float* __restrict__ src, __half* __restrict__ dst,
                                  int rows, int cols, long long lds, long long ldd)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const long long c = blockIdx.y;
    if (r < rows && c < cols) dst[c * ldd + r] = __float2half_rn(src[c * lds + r]);
}

__global__ void f16_to_f32_kernel(const __half* __restrict__ src, float* __restrict__ dst,
                                  int rows, int cols, long long lds, long long ldd)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const long long c = blockIdx.y;
    if (r < rows && c < cols) dst[c * ldd + r] = __half2float(src[c * lds + r]);
}

// max |A(i,i)| as ordered float bits (non-negative floats order like uints).
__global__ void diag_absmax_kernel(const float* A, int n, long long lda, unsigned int* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float v = 0.f;
    if (i < n) v = fabsf(A[(long long)i * lda + i]);
    for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(v));
}

// Scale the lower triangle (diagonal included) of column blockIdx.x.
__global__ void scale_lower_kernel(float* A, int n, long long lda, const unsigned int* maxbits,
                                   int inverse)
{
    const long long c = blockIdx.x;
    const float mx = __uint_as_float(*maxbits);
    if (!(mx > 0.f)) return;
    const float f = inverse ? sqrtf(mx / HDBF_SCALE_TARGET) : HDBF_SCALE_TARGET / mx;
    for (long long r = c + threadIdx.x; r < n; r += blockDim.x) A[c * lda + r] *= f;
}

__device__ __forceinline__ unsigned long long splitmix_finalize(unsigned long long x)
{
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

__global__ void fill_uniform_kernel(float* x, unsigned long long count, unsigned long long seed,
                                    unsigned long long offset)
{
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         i < count; i += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long h = seed * 0x9E3779B97F4A7C15ull + (offset + i + 1ull) * 0xD1B54A32D192ED03ull;
        h = splitmix_finalize(h);
        const unsigned int top = (unsigned int)(h >> 40);  // 24 bits
        x[i] = (float)((double)top / 8388608.0 - 1.0);
    }
}

}  // namespace

hdbf_status add_damping(cudaStream_t s, float* A, int n, long long lda, float lambda)
{
    if (n <= 0) return HDBF_STATUS_SUCCESS;
    add_damping_kernel<float><<<(n + 255) / 256, 256, 0, s>>>(A, n, lda, lambda);
    return cudaGetLastError() == cudaSuccess ? HDBF_STATUS_SUCCESS : HDBF_STATUS_CUDA_ERROR;
}

hdbf_status fill_uniform(hdbf_context* ctx, float* x, size_t count, uint64_t seed,
                         uint64_t offset)
{
    if (count == 0) return HDBF_STATUS_SUCCESS;
    const unsigned long long blocks = (count + 255) / 256;
    const unsigned grid = (unsigned)(blocks < 65535ull * 16 ? blocks : 65535ull * 16);
    fill_uniform_kernel<<<grid, 256, 0, ctx->stream>>>(x, count, seed, offset);
    ctx->launches++;
    return last_cuda(ctx);
}

}  // namespace hdbf

using namespace hdbf;

extern "C" {

void launch_add_damping(float* A, int n, int lda, float lambda, cudaStream_t stream)
{
    if (!A || n <= 0) return;
    add_damping_kernel<float><<<(n + 255) / 256, 256, 0, stream>>>(A, n, lda, lambda);
}

void launch_add_damping_double(double* A, int n, int lda, double lambda, cudaStream_t stream)
{
    if (!A || n <= 0) return;
    add_damping_kernel<double><<<(n + 255) / 256, 256, 0, stream>>>(A, n, lda, lambda);
}

void launch_fp32_to_fp16(const float* src, void* dst, int rows, int cols, int ld_src,
                         int ld_dst, cudaStream_t stream)
{
    if (!src || !dst || rows <= 0 || cols <= 0) return;
    dim3 grid((rows + 255) / 256, cols);
    f32_to_f16_kernel<<<grid, 256, 0, stream>>>(src, static_cast<__half*>(dst), rows, cols,
                                                ld_src, ld_dst);
}

void launch_fp16_to_fp32(const void* src, float* dst, int rows, int cols, int ld_src,
                         int ld_dst, cudaStream_t stream)
{
    if (!src || !dst || rows <= 0 || cols <= 0) return;
    dim3 grid((rows + 255) / 256, cols);
    f16_to_f32_kernel<<<grid, 256, 0, stream>>>(static_cast<const __half*>(src), dst, rows,
                                                cols, ld_src, ld_dst);
}

void launch_auto_scale(float* A, int n, int lda, unsigned int* d_max_val, bool inverse,
                       cudaStream_t stream)
{
    if (!A || !d_max_val || n <= 0) return;
    if (!inverse) {
        cudaMemsetAsync(d_max_val, 0, sizeof(unsigned int), stream);
        diag_absmax_kernel<<<(n + 255) / 256, 256, 0, stream>>>(A, n, lda, d_max_val);
    }
    scale_lower_kernel<<<n, 256, 0, stream>>>(A, n, lda, d_max_val, inverse ? 1 : 0);
}

}  // extern "C"
