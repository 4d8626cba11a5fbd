// Test-infrastructure shim: exposes the reference's own header-only CPU FP64
// residual (include/utils/benchmark/cpu_fp64_residual.h, compiled in place from
// the reference tree) through plain C symbols so the tests can cross-check the
// C restatement in residual.c against it. Built only into oracle/_ref/.
#include "utils/benchmark/cpu_fp64_residual.h"

#include <limits>
#include <stdexcept>

namespace {
template <typename F>
double guarded(F&& f, int* err)
{
    *err = 0;
    try {
        return f();
    } catch (const std::invalid_argument&) {
        *err = 1;
        return std::numeric_limits<double>::quiet_NaN();
    }
}
}  // namespace

extern "C" {
double ref_potrf_residual_f32(const float* L, const float* A, int n, int lda, int tile, int* err)
{
    return guarded([&] { return benchmark_residual::potrf_cpu_fp64_full(L, A, n, lda, tile); }, err);
}
double ref_potrf_residual_f64(const double* L, const double* A, int n, int lda, int tile, int* err)
{
    return guarded([&] { return benchmark_residual::potrf_cpu_fp64_full(L, A, n, lda, tile); }, err);
}
double ref_getrf_residual_f32(const float* LU, const float* A, const int* ipiv, int n, int lda,
                              int pivoting, int tile, int* err)
{
    return guarded([&] {
        return benchmark_residual::getrf_cpu_fp64_full(LU, A, ipiv, n, lda, pivoting != 0, tile);
    }, err);
}
double ref_getrf_residual_f64(const double* LU, const double* A, const int* ipiv, int n, int lda,
                              int pivoting, int tile, int* err)
{
    return guarded([&] {
        return benchmark_residual::getrf_cpu_fp64_full(LU, A, ipiv, n, lda, pivoting != 0, tile);
    }, err);
}
}
