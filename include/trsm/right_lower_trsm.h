/*
 * Right, lower, transposed, non-unit triangular solve B <- B * L^{-T}, FP32.
 * Drop-in for reference include/trsm/right_lower_trsm.h:9-15
 * (src/trsm/right_lower_trsm.cpp:9-55).  B is rows x cols, L is cols x cols.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void trsm_right_lower_transpose(hdbf_handle handle, int rows, int cols, const float* A,
                                int lda, float* B, int ldb);

#ifdef __cplusplus
}
#endif
