/*
 * Source-compatibility shim for code written against the reference's
 * rocBLAS-typed headers: maps the few rocBLAS/HIP type names that appear in the
 * reference's public signatures onto this library's types.
 */
#pragma once

#include "hdbf/hdbf.h"

typedef hdbf_handle rocblas_handle;

/* rocblas_operation values as used by launch_mixed_gemm
 * (reference include/gemm/mixed_gemm.h:10-22). */
typedef enum rocblas_operation_ {
    rocblas_operation_none = 111,
    rocblas_operation_transpose = 112,
    rocblas_operation_conjugate_transpose = 113
} rocblas_operation;
