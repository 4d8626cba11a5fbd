// Handle, stream pool, workspace arena and status plumbing (host C++).
#include <cstdlib>
#include <cstring>
#include <new>

#include "internal.h"

namespace hdbf {

hdbf_status last_cuda(hdbf_context* ctx)
{
    cudaError_t e = cudaGetLastError();
    (void)ctx;
    return e == cudaSuccess ? HDBF_STATUS_SUCCESS : HDBF_STATUS_CUDA_ERROR;
}

void* workspace(hdbf_context* ctx, size_t bytes, hdbf_status* st)
{
    *st = HDBF_STATUS_SUCCESS;
    if (bytes <= ctx->ws_bytes) return ctx->ws;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cs) == cudaSuccess &&
        cs != cudaStreamCaptureStatusNone) {
        *st = HDBF_STATUS_WORKSPACE_TOO_SMALL;
        return nullptr;
    }
    if (ctx->ws) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->ws);
        ctx->ws = nullptr;
        ctx->ws_bytes = 0;
    }
    size_t want = align_up(bytes, size_t(1) << 20);
    if (cudaMalloc(&ctx->ws, want) != cudaSuccess) {
        cudaGetLastError();
        ctx->ws = nullptr;
        *st = HDBF_STATUS_ALLOC_FAILED;
        return nullptr;
    }
    ctx->ws_bytes = want;
    return ctx->ws;
}

static cudaEvent_t pool_event(hdbf_context* ctx)
{
    if (ctx->ev_used == ctx->ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ctx->ev_pool.push_back(e);
    }
    return ctx->ev_pool[ctx->ev_used++];
}

ProfScope::ProfScope(hdbf_context* ctx, int cls, double flops, double bytes) : ctx_(ctx)
{
    if (!ctx || !ctx->profiling) return;
    cudaEvent_t a = pool_event(ctx), b = pool_event(ctx);
    if (!a || !b) return;
    cudaEventRecord(a, ctx->stream);
    idx_ = static_cast<int>(ctx->prof.size());
    ctx->prof.push_back(ProfRec{cls, a, b, flops, bytes});
}

ProfScope::~ProfScope()
{
    if (idx_ < 0) return;
    cudaEventRecord(ctx_->prof[idx_].b, ctx_->stream);
}

}  // namespace hdbf

using namespace hdbf;

extern "C" {

hdbf_status hdbf_create(hdbf_handle* handle)
{
    if (!handle) return HDBF_STATUS_INVALID_VALUE;
    *handle = nullptr;
    hdbf_context* ctx = new (std::nothrow) hdbf_context();
    if (!ctx) return HDBF_STATUS_ALLOC_FAILED;
    if (cudaGetDevice(&ctx->device) != cudaSuccess) {
        delete ctx;
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    ctx->max_smem_optin = static_cast<size_t>(optin);
    if (cudaMalloc(&ctx->dev_small, kSmallInts * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return HDBF_STATUS_ALLOC_FAILED;
    }
    cudaMemset(ctx->dev_small, 0, kSmallInts * sizeof(int));
    cudaDeviceSynchronize();
    *handle = ctx;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_destroy(hdbf_handle h)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    cudaStreamSynchronize(h->stream);
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    if (h->ws) cudaFree(h->ws);
    if (h->dev_small) cudaFree(h->dev_small);
    delete h;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_set_stream(hdbf_handle h, void* stream)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    h->stream = static_cast<cudaStream_t>(stream);
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_get_stream(hdbf_handle h, void** stream)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (!stream) return HDBF_STATUS_INVALID_VALUE;
    *stream = h->stream;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_get_last_status(hdbf_handle h)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    return h->last_status;
}

const char* hdbf_status_string(hdbf_status s)
{
    switch (s) {
    case HDBF_STATUS_SUCCESS: return "success";
    case HDBF_STATUS_INVALID_HANDLE: return "invalid handle";
    case HDBF_STATUS_INVALID_VALUE: return "invalid value";
    case HDBF_STATUS_ALLOC_FAILED: return "device allocation failed";
    case HDBF_STATUS_CUDA_ERROR: return "CUDA error";
    case HDBF_STATUS_NOT_SUPPORTED: return "not supported";
    case HDBF_STATUS_TIMEOUT: return "device-side wait timed out";
    case HDBF_STATUS_WORKSPACE_TOO_SMALL: return "workspace too small during stream capture";
    }
    return "unknown status";
}

size_t hdbf_workspace_bytes_for(int n)
{
    if (n < 1) n = 1;
    // coop panel scratch + compose moves (src, tgt, gperm: 3 n ints) +
    // a column-tiled swap buffer (64 columns x n floats) + slack.
    size_t b = getf2_coop_scratch_bytes();
    b += 3 * align_up(size_t(n) * sizeof(int), 256);
    b += align_up(size_t(64) * size_t(n) * sizeof(float), 256);
    b += size_t(1) << 20;
    return b;
}

hdbf_status hdbf_reserve_workspace(hdbf_handle h, size_t bytes)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    hdbf_status st;
    workspace(h, bytes, &st);
    return st;
}

hdbf_status hdbf_check_device_errors(hdbf_handle h)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    int err = 0;
    if (cudaMemcpy(&err, h->dev_small + kSmallErr, sizeof(int), cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    if (err != 0) {
        // Clear the error word and re-arm the grid barrier for later launches.
        cudaMemset(h->dev_small, 0, kSmallInts * sizeof(int));
        cudaDeviceSynchronize();
        return err == kErrTimeout ? HDBF_STATUS_TIMEOUT : HDBF_STATUS_INVALID_VALUE;
    }
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_stream_pool_create(int num_streams, StreamPool** pool)
{
    if (!pool || num_streams < 1) return HDBF_STATUS_INVALID_VALUE;
    hdbf_stream_pool* p = new (std::nothrow) hdbf_stream_pool();
    if (!p) return HDBF_STATUS_ALLOC_FAILED;
    p->streams = new (std::nothrow) cudaStream_t[num_streams];
    if (!p->streams) {
        delete p;
        return HDBF_STATUS_ALLOC_FAILED;
    }
    for (int i = 0; i < num_streams; ++i) {
        if (cudaStreamCreateWithFlags(&p->streams[i], cudaStreamNonBlocking) != cudaSuccess) {
            for (int j = 0; j < i; ++j) cudaStreamDestroy(p->streams[j]);
            delete[] p->streams;
            delete p;
            cudaGetLastError();
            return HDBF_STATUS_CUDA_ERROR;
        }
    }
    p->count = num_streams;
    *pool = p;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_stream_pool_destroy(StreamPool* pool)
{
    if (!pool) return HDBF_STATUS_INVALID_VALUE;
    for (int i = 0; i < pool->count; ++i) cudaStreamDestroy(pool->streams[i]);
    delete[] pool->streams;
    delete pool;
    return HDBF_STATUS_SUCCESS;
}

int hdbf_stream_pool_size(const StreamPool* pool) { return pool ? pool->count : 0; }

hdbf_status hdbf_fill_uniform(hdbf_handle h, float* x, size_t count, unsigned long long seed,
                              unsigned long long offset)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (!x && count) return HDBF_STATUS_INVALID_VALUE;
    return fill_uniform(h, x, count, seed, offset);
}

unsigned long long hdbf_launch_count(hdbf_handle h) { return h ? h->launches : 0ull; }

hdbf_status hdbf_profile_begin(hdbf_handle h)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    h->prof.clear();
    h->ev_used = 0;
    h->profiling = true;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_profile_end(hdbf_handle h, int max_classes, double* ms, double* flops,
                             double* bytes, unsigned long long* launches)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    h->profiling = false;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    for (int c = 0; c < max_classes; ++c) {
        if (ms) ms[c] = 0.0;
        if (flops) flops[c] = 0.0;
        if (bytes) bytes[c] = 0.0;
        if (launches) launches[c] = 0;
    }
    for (const ProfRec& r : h->prof) {
        if (r.cls < 0 || r.cls >= max_classes) continue;
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        if (ms) ms[r.cls] += t;
        if (flops) flops[r.cls] += r.flops;
        if (bytes) bytes[r.cls] += r.bytes;
        if (launches) launches[r.cls] += 1;
    }
    h->prof.clear();
    h->ev_used = 0;
    return HDBF_STATUS_SUCCESS;
}

const char* hdbf_profile_class_name(int cls)
{
    static const char* names[kNumClasses] = {"sgemm_sub_kernel", "potf2_kernel",
                                             "trsm_rlt_kernel", "trsm_llu_kernel",
                                             "getf2_coop_kernel", "compose_swaps_kernel",
                                             "apply_moves", "other"};
    return (cls >= 0 && cls < kNumClasses) ? names[cls] : "unknown";
}

int hdbf_profile_num_classes(void) { return kNumClasses; }

}  // extern "C"
