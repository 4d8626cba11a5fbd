/*
 * Iterative right-looking right/lower/transposed TRSM, FP32.
 * Drop-in for reference include/trsm/iterative_trsm.h:8-11
 * (src/trsm/iterative_trsm.cpp:6-60): nb-wide column panels, each solved then
 * used to update the remaining columns.
 */
#pragma once
#include "hdbf/hdbf.h"

#ifdef __cplusplus
extern "C" {
#endif

void iterative_trsm_right_looking(hdbf_handle handle, float* A, int lda, float* B, int ldb,
                                  int n, int m, int nb);

#ifdef __cplusplus
}
#endif
