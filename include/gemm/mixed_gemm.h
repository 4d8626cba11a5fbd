/*
 * Mixed-precision GEMM C = alpha * op(A) * op(B) + beta * C with FP32 operands
 * in memory, FP16 tensor-core products (tcgen05, kind::f16) and FP32
 * accumulation and FP32 C.
 * Drop-in for reference include/gemm/mixed_gemm.h:10-22
 * (src/gemm/mixed_gemm.cpp:8-96); the reference stores C in FP16 and
 * allocates per call, this version keeps C in FP32 and uses the handle's
 * workspace.  The `handle` argument supplies the workspace; `stream` is the
 * stream the work is enqueued on.
 */
#pragma once
#include <cuda_runtime_api.h>
#include "hdbf/hdbf.h"
#include "hdbf/rocblas_compat.h"

#ifdef __cplusplus
extern "C" {
#endif

void launch_mixed_gemm(hdbf_handle handle, cudaStream_t stream, rocblas_operation transA,
                       rocblas_operation transB, int m, int n, int k, float alpha,
                       const float* A_f32, int lda, const float* B_f32, int ldb, float beta,
                       float* C_f32, int ldc);

#ifdef __cplusplus
}
#endif
