/*
 * Column-major FP32 <-> FP16 copies with independent leading dimensions.
 * Drop-in for reference include/kernels/fp16_convert.h:11-31
 * (src/kernels/fp16_convert.hip:12-129).  The FP16 buffers are IEEE binary16
 * (`__half` in CUDA), passed as void* so the header needs no fp16 include.
 */
#pragma once
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

void launch_fp32_to_fp16(const float* src, void* dst, int rows, int cols, int ld_src,
                         int ld_dst, cudaStream_t stream);
void launch_fp16_to_fp32(const void* src, float* dst, int rows, int cols, int ld_src,
                         int ld_dst, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
