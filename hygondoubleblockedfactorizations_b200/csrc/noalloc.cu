// Allocation-free variant of trsm_right_lower_transpose.
//
// Some callers cannot allocate device memory at the point where they need a
// triangular solve: real-time or embedded services whose device memory is
// fixed at start-up, and host libraries that may hand out only caller-owned
// buffers.  The regular entry point
// allocates a per-handle workspace (and the handle itself allocates on
// creation); this one takes a bare stream and keeps its only scratch -- the
// inverted 64x64 diagonal blocks of L -- in a fixed-size device array that is
// part of the library image.
#include <mutex>

#include "internal.h"
#include "trsm/right_lower_trsm.h"

namespace hdbf {
namespace {

constexpr int kDiagLeaf = 64;
constexpr int kMaxDevices = 64;

// Scratch for the inverted diagonal blocks: HDBF_NOALLOC_TRSM_MAX_COLS / 64
// blocks of 64 x 64 floats (1 MiB).  Every GPU that loads the library holds
// this array until the process exits.
static __device__ __align__(256) float g_noalloc_inv[HDBF_NOALLOC_TRSM_MAX_COLS * kDiagLeaf];

// Device address of g_noalloc_inv per device.  In host code the symbol names
// a host-side stand-in, so the address must be queried with the device
// current and passed to the kernels explicitly.
float* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

hdbf_status scratch_for_current_device(float** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_inv) != cudaSuccess || !p) {
            cudaGetLastError();
            return HDBF_STATUS_CUDA_ERROR;
        }
        g_scratch_addr[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_addr[dev];
    return HDBF_STATUS_SUCCESS;
}

inline int split_at(int n)
{
    int h = (n / 2 + kDiagLeaf - 1) / kDiagLeaf * kDiagLeaf;
    if (h <= 0 || h >= n) h = n > kDiagLeaf ? n - kDiagLeaf : 1;
    return h;
}

// B(rows x cols) <- B * L^{-T} with the block inverses already in `inv`:
// column halves, GEMM update between them, leaves applied with the inverses.
hdbf_status rlt_recurse(hdbf_context* ctx, int rows, int cols, const float* L, long long ldl,
                        float* B, long long ldb, const float* inv)
{
    if (cols <= kDiagLeaf) return rlt_apply(ctx, rows, cols, inv, B, ldb);
    const int c1 = split_at(cols);
    const int c2 = cols - c1;
    HDBF_TRY(rlt_recurse(ctx, rows, c1, L, ldl, B, ldb, inv));
    HDBF_TRY(sgemm_sub(ctx, false, false, rows, c2, c1, B, ldb, L + c1, ldl,
                       B + (long long)c1 * ldb, ldb));
    return rlt_recurse(ctx, rows, c2, L + (long long)c1 * ldl + c1, ldl, B + (long long)c1 * ldb,
                       ldb, inv + (long long)(c1 / kDiagLeaf) * kDiagLeaf * kDiagLeaf);
}

}  // namespace
}  // namespace hdbf

using namespace hdbf;

extern "C" hdbf_status trsm_right_lower_transpose_noalloc(int rows, int cols, const float* A,
                                                          int lda, float* B, int ldb,
                                                          cudaStream_t stream)
{
    if (rows < 0 || cols < 0) return HDBF_STATUS_INVALID_VALUE;
    if (cols > HDBF_NOALLOC_TRSM_MAX_COLS) return HDBF_STATUS_INVALID_VALUE;
    if (rows == 0 || cols == 0) return HDBF_STATUS_SUCCESS;
    if (!A || !B || lda < cols || ldb < rows) return HDBF_STATUS_INVALID_VALUE;
    float* inv = nullptr;
    HDBF_TRY(scratch_for_current_device(&inv));
    // A stack context carries only the stream; none of the kernels launched
    // below touches its workspace fields, and profiling stays off.
    hdbf_context ctx;
    ctx.stream = stream;
    HDBF_TRY(tri_inv64(&ctx, cols, A, lda, false, inv));
    return rlt_recurse(&ctx, rows, cols, A, lda, B, ldb, inv);
}
