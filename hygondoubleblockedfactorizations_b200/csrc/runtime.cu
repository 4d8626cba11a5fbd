#include <algorithm>
// Handle, stream pool, workspace arena and status plumbing (host C++).
#include <cstdio>
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

static int fitting_order(size_t bytes);

void* workspace(hdbf_context* ctx, size_t bytes, hdbf_status* st)
{
    *st = HDBF_STATUS_SUCCESS;
    if (bytes <= ctx->ws_bytes && ctx->ws) return ctx->ws;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cs) == cudaSuccess &&
        cs != cudaStreamCaptureStatusNone) {
        *st = HDBF_STATUS_WORKSPACE_TOO_SMALL;
        return nullptr;
    }
    graph_cache_clear(ctx);  // cached graphs point into the old arena
    if (ctx->ws) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->ws);
        ctx->ws = nullptr;
        ctx->ws_bytes = 0;
        ctx->ws_n = 0;
    }
    size_t want = align_up(bytes, size_t(1) << 20);
    if (cudaMalloc(&ctx->ws, want) != cudaSuccess) {
        cudaGetLastError();
        ctx->ws = nullptr;
        *st = HDBF_STATUS_ALLOC_FAILED;
        return nullptr;
    }
    ctx->ws_bytes = want;
    ctx->ws_n = fitting_order(want);
    // Exchange slots must never hold a stale tag that matches a live one:
    // clear the whole arena on every (re)allocation.
    cudaMemset(ctx->ws, 0, want);
    cudaDeviceSynchronize();
    return ctx->ws;
}

void* mixed_arena(hdbf_context* ctx, size_t bytes, hdbf_status* st)
{
    *st = HDBF_STATUS_SUCCESS;
    if (bytes <= ctx->mix_bytes && ctx->mix) return ctx->mix;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cs) == cudaSuccess &&
        cs != cudaStreamCaptureStatusNone) {
        *st = HDBF_STATUS_WORKSPACE_TOO_SMALL;
        return nullptr;
    }
    graph_cache_clear(ctx);  // cached graphs point into the old arena
    if (ctx->mix) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->mix);
        ctx->mix = nullptr;
        ctx->mix_bytes = 0;
    }
    const size_t want = align_up(bytes, size_t(1) << 20);
    if (cudaMalloc(&ctx->mix, want) != cudaSuccess) {
        cudaGetLastError();
        ctx->mix = nullptr;
        *st = HDBF_STATUS_ALLOC_FAILED;
        return nullptr;
    }
    ctx->mix_bytes = want;
    return ctx->mix;
}

WsLayout ws_layout(int n)
{
    if (n < 64) n = 64;
    WsLayout L;
    size_t off = 0;
    L.coop = off;
    off += getf2_coop_scratch_bytes();
    L.inv = off;  // whole 64x64 blocks, the last one padded
    off += align_up((size_t)(n + 63) / 64 * 64 * 64 * sizeof(float), 256);
    L.perm = off;
    off += align_up((size_t)n * sizeof(int), 256);
    L.coop64 = off;
    off += getf2_coop64_scratch_bytes();
    L.src = off;
    off += align_up((size_t)n * sizeof(int), 256);
    L.tgt = off;
    off += align_up((size_t)n * sizeof(int), 256);
    L.gperm = off;
    off += align_up((size_t)n * sizeof(int), 256);
    L.temp = off;
    off += align_up((size_t)64 * n * sizeof(float), 256);
    L.skinny = off;
    off += align_up(skinny_partial_floats(n) * sizeof(float), 256);
    L.wave = off;
    off += wave_scratch_bytes(n);
    L.split = off;
    off += align_up(2 * kSplitFloats * sizeof(float), 256);
    L.total = off;
    return L;
}

static int fitting_order(size_t bytes)
{
    if (ws_layout(64).total > bytes) return 0;
    int lo = 64, hi = 1 << 24;
    while (lo < hi) {
        const int mid = lo + (hi - lo + 1) / 2;
        if (ws_layout(mid).total <= bytes) lo = mid; else hi = mid - 1;
    }
    return lo;
}

hdbf_status ensure_ws(hdbf_context* ctx, int n)
{
    if (n <= ctx->ws_n && ctx->ws) return HDBF_STATUS_SUCCESS;
    const int want = n > ctx->ws_n ? n : ctx->ws_n;
    hdbf_status st;
    workspace(ctx, ws_layout(want).total, &st);
    return st;
}

float* ws_coop(hdbf_context* ctx)
{
    return reinterpret_cast<float*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).coop);
}
float* ws_inv(hdbf_context* ctx)
{
    return reinterpret_cast<float*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).inv);
}
double* ws_coop64(hdbf_context* ctx)
{
    return reinterpret_cast<double*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).coop64);
}

int* ws_perm(hdbf_context* ctx)
{
    return reinterpret_cast<int*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).perm);
}

hdbf_status ensure_lookahead(hdbf_context* ctx)
{
    if (ctx->la_stream) return HDBF_STATUS_SUCCESS;
    if (ctx->capturing) return HDBF_STATUS_NOT_SUPPORTED;
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    for (int i = 0; i < kLaEvents; ++i) {
        if (cudaEventCreateWithFlags(&ctx->la_ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            for (int j = 0; j < i; ++j) cudaEventDestroy(ctx->la_ev[j]);
            cudaStreamDestroy(s);
            return HDBF_STATUS_CUDA_ERROR;
        }
    }
    ctx->la_stream = s;
    return HDBF_STATUS_SUCCESS;
}

int* ws_src(hdbf_context* ctx)
{
    return reinterpret_cast<int*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).src);
}
int* ws_tgt(hdbf_context* ctx)
{
    return reinterpret_cast<int*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).tgt);
}
int* ws_gperm(hdbf_context* ctx)
{
    return reinterpret_cast<int*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).gperm);
}
float* ws_temp(hdbf_context* ctx)
{
    return reinterpret_cast<float*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).temp);
}
float* ws_wave(hdbf_context* ctx)
{
    return reinterpret_cast<float*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).wave);
}
float* ws_skinny(hdbf_context* ctx)
{
    return reinterpret_cast<float*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).skinny);
}
float* ws_split(hdbf_context* ctx)
{
    float* base =
        reinterpret_cast<float*>(static_cast<char*>(ctx->ws) + ws_layout(ctx->ws_n).split);
    return (ctx->la_stream && ctx->stream == ctx->la_stream) ? base + kSplitFloats : base;
}

ProfScope::ProfScope(hdbf_context* ctx, int cls, double flops, double bytes, int m, int n,
                     int k)
    : ctx_(ctx)
{
    if (!ctx || !ctx->profiling) return;
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        cudaGetLastError();
        if (a) cudaEventDestroy(a);
        return;
    }
    // Under capture the record must become a real event node of the graph
    // (a plain record would only express a dependency).
    cudaEventRecordWithFlags(a, ctx->stream, ctx->capturing ? cudaEventRecordExternal : 0);
    idx_ = static_cast<int>(ctx->prof.size());
    ctx->prof.push_back(ProfRec{cls, a, b, flops, bytes, m, n, k, ctx->stage, ctx->stage_call});
}

ProfScope::~ProfScope()
{
    if (idx_ < 0) return;
    cudaEventRecordWithFlags(ctx_->prof[idx_].b, ctx_->stream,
                             ctx_->capturing ? cudaEventRecordExternal : 0);
}

static void destroy_records(std::vector<ProfRec>& v)
{
    for (ProfRec& r : v) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    v.clear();
}

// ------------------------------------------------------------------ graphs
constexpr size_t kMaxGraphs = 12;

void graph_cache_clear(hdbf_context* ctx)
{
    for (GraphEntry& e : ctx->graphs) {
        if (e.exec) cudaGraphExecDestroy(e.exec);
        destroy_records(e.prof);
    }
    ctx->graphs.clear();
    ctx->prof_graph_ids.clear();
}

bool graph_can_capture(hdbf_context* ctx)
{
    if (!ctx->use_graphs || ctx->capturing) return false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return cs == cudaStreamCaptureStatusNone;  // the caller is not capturing us itself
}

GraphEntry* graph_find(hdbf_context* ctx, const std::vector<long long>& key)
{
    for (GraphEntry& e : ctx->graphs)
        if (e.key == key) return &e;
    return nullptr;
}

hdbf_status graph_capture_begin(hdbf_context* ctx, cudaStream_t* saved)
{
    if (!ctx->cap_stream &&
        cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    if (cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    *saved = ctx->stream;
    ctx->stream = ctx->cap_stream;
    ctx->capturing = true;
    ctx->la_used = false;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status graph_capture_end(hdbf_context* ctx, cudaStream_t saved, hdbf_status body_status,
                              const std::vector<long long>& key, size_t prof_mark,
                              unsigned long long launches_before)
{
    const unsigned long long kernels = ctx->launches - launches_before;
    ctx->launches = launches_before;  // counted when the graph actually runs
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(ctx->cap_stream, &graph);
    ctx->stream = saved;
    ctx->capturing = false;
    std::vector<ProfRec> recs(ctx->prof.begin() + prof_mark, ctx->prof.end());
    ctx->prof.resize(prof_mark);
    if (ce != cudaSuccess || !graph) {
        cudaGetLastError();
        if (graph) cudaGraphDestroy(graph);
        destroy_records(recs);
        ctx->use_graphs = false;  // this work cannot be captured here: stay eager
        return HDBF_STATUS_NOT_SUPPORTED;
    }
    if (body_status != HDBF_STATUS_SUCCESS) {
        cudaGraphDestroy(graph);
        destroy_records(recs);
        return body_status;
    }
    cudaGraphExec_t exec = nullptr;
    // A look-ahead graph keeps the priorities its kernel nodes were captured
    // with (the panel chain's high-priority stream), not the launch stream's.
    const unsigned long long iflags = ctx->la_used ? cudaGraphInstantiateFlagUseNodePriority : 0;
    ctx->la_used = false;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, iflags);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        cudaGetLastError();
        destroy_records(recs);
        ctx->use_graphs = false;
        return HDBF_STATUS_NOT_SUPPORTED;
    }
    if (ctx->graphs.size() >= kMaxGraphs) {  // evict the least recently used
        size_t lru = 0;
        for (size_t i = 1; i < ctx->graphs.size(); ++i)
            if (ctx->graphs[i].last_use < ctx->graphs[lru].last_use) lru = i;
        cudaGraphExecDestroy(ctx->graphs[lru].exec);
        destroy_records(ctx->graphs[lru].prof);
        ctx->graphs.erase(ctx->graphs.begin() + lru);
    }
    GraphEntry e;
    e.key = key;
    e.exec = exec;
    e.prof = std::move(recs);
    e.id = ++ctx->graph_clock;
    e.kernels = kernels;
    ctx->graphs.push_back(std::move(e));
    return graph_launch(ctx, &ctx->graphs.back());
}

hdbf_status graph_launch(hdbf_context* ctx, GraphEntry* e)
{
    e->last_use = ++ctx->graph_clock;
    if (ctx->profiling && !e->prof.empty()) ctx->prof_graph_ids.push_back(e->id);
    if (cudaGraphLaunch(e->exec, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    ctx->launches += e->kernels;
    return HDBF_STATUS_SUCCESS;
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
    configure_getrf_kernels(ctx);
    ctx->cluster_max = configure_cluster_panel(ctx);
    if (const char* pk = std::getenv("HDBF_PANEL_KERNEL")) {  // default panel kernel
        const int v = std::atoi(pk);
        if (v >= 0 && v <= 2) ctx->panel_mode = v;
    }
    if (const char* pl = std::getenv("HDBF_PANEL_LEAF")) {  // default panel leaf width
        const int v = std::atoi(pl);
        if (v == 32 || v == 64 || v == 128) ctx->panel_leaf = v;
    }
    if (const char* pr = std::getenv("HDBF_PANEL_ROWS")) {  // rows per panel CTA
        const int v = std::atoi(pr);
        if (v >= 64 && v <= 4096) ctx->panel_rows = v;
    }
    if (const char* la = std::getenv("HDBF_LOOKAHEAD")) ctx->lookahead = std::atoi(la) != 0;
    if (const char* tk = std::getenv("HDBF_TC_KERNEL")) ctx->tc_kernel = std::atoi(tk) != 0;
    configure_tc_kernels(ctx);
    configure_trsm_block_kernels(ctx);
    configure_solve_kernels(ctx);
    configure_batched_kernels(ctx);
    configure_fp64_kernels(ctx);
    const int one = 1;  // exchange epoch starts at 1: zeroed slots never match
    cudaMemcpy(ctx->dev_small + kSmallEpoch, &one, sizeof(int), cudaMemcpyHostToDevice);
    cudaDeviceSynchronize();
    *handle = ctx;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_destroy(hdbf_handle h)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    cudaStreamSynchronize(h->stream);
    graph_cache_clear(h);
    destroy_records(h->prof);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->la_stream) {
        cudaStreamSynchronize(h->la_stream);
        for (int i = 0; i < kLaEvents; ++i) cudaEventDestroy(h->la_ev[i]);
        cudaStreamDestroy(h->la_stream);
    }
    if (h->ws) cudaFree(h->ws);
    if (h->dev_small) cudaFree(h->dev_small);
    if (h->mix) cudaFree(h->mix);
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

size_t hdbf_workspace_bytes_for(int n) { return ws_layout(n < 1 ? 1 : n).total; }

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
        // Clear the error word and the exchange counters, and advance the
        // epoch past every sequence number a timed-out launch may have left.
        unsigned epoch = 0;
        cudaMemcpy(&epoch, h->dev_small + kSmallEpoch, sizeof(int), cudaMemcpyDeviceToHost);
        cudaMemset(h->dev_small, 0, kSmallInts * sizeof(int));
        if (h->ws) cudaMemset(h->ws, 0, h->ws_bytes);  // exchange words with the counters
        epoch += 2;
        cudaMemcpy(h->dev_small + kSmallEpoch, &epoch, sizeof(int), cudaMemcpyHostToDevice);
        cudaMemcpy(h->dev_small + kSmallSpin, &h->spin_limit, sizeof(unsigned),
                   cudaMemcpyHostToDevice);
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
    destroy_records(h->prof);
    h->prof_graph_ids.clear();
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
    // HDBF_PROFILE_CSV=<path>: also append one line per launch (class, ms,
    // flops, bytes, m, n, k) for offline analysis.
    const char* csv_path = std::getenv("HDBF_PROFILE_CSV");
    FILE* csv = csv_path ? std::fopen(csv_path, "a") : nullptr;
    for (int st = 0; st < kNumStages; ++st) {
        h->stage_ms[st] = 0.0;
        h->stage_flops[st] = 0.0;
        h->stage_calls[st] = 0;
    }
    std::vector<std::pair<int, unsigned>> calls_seen;
    auto add = [&](const ProfRec& r) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        if (r.stage > 0 && r.stage < kNumStages) {
            h->stage_ms[r.stage] += t;
            h->stage_flops[r.stage] += r.flops;
            const std::pair<int, unsigned> key(r.stage, r.call);
            if (std::find(calls_seen.begin(), calls_seen.end(), key) == calls_seen.end()) {
                calls_seen.push_back(key);
                h->stage_calls[r.stage] += 1;
            }
        }
        if (r.cls < 0 || r.cls >= max_classes) return;
        if (csv)
            std::fprintf(csv, "%s,%.6f,%.6g,%.6g,%d,%d,%d,%s\n", hdbf_profile_class_name(r.cls), t,
                         r.flops, r.bytes, r.m, r.n, r.k, hdbf_profile_stage_name(r.stage));
        if (ms) ms[r.cls] += t;
        if (flops) flops[r.cls] += r.flops;
        if (bytes) bytes[r.cls] += r.bytes;
        if (launches) launches[r.cls] += 1;
    };
    for (const ProfRec& r : h->prof) add(r);
    // Graphs replayed while profiling: their event nodes hold the timings of
    // the latest replay (each graph counted once).
    std::vector<unsigned long long> seen;
    for (unsigned long long id : h->prof_graph_ids) {
        bool dup = false;
        for (unsigned long long s2 : seen) dup = dup || s2 == id;
        if (dup) continue;
        seen.push_back(id);
        for (const GraphEntry& e : h->graphs)
            if (e.id == id)
                for (const ProfRec& r : e.prof) add(r);
    }
    if (csv) std::fclose(csv);
    destroy_records(h->prof);
    h->prof_graph_ids.clear();
    return HDBF_STATUS_SUCCESS;
}

const char* hdbf_profile_class_name(int cls)
{
    static const char* names[kNumClasses] = {"sgemm_sub_kernel", "potf2_kernel",
                                             "rlt_apply_kernel", "llu_apply_kernel",
                                             "getf2_panel_kernel", "compose_swaps_kernel",
                                             "apply_moves", "tri_inv64_kernel",
                                             "tc_gemm_kernels", "convert16_kernels",
                                             "ir_fp64_kernels", "other",
                                             "trsv_wave_kernel", "sgemm_skinny_kernel",
                                             "batched_factor_solve_kernel",
                                             "selector_mlp_kernels", "potrf_block_kernel"};
    return (cls >= 0 && cls < kNumClasses) ? names[cls] : "unknown";
}

int hdbf_profile_num_classes(void) { return kNumClasses; }

const char* hdbf_profile_stage_name(int stage)
{
    static const char* names[kNumStages] = {
        "none", "POTRF", "TRSM", "Inner GEMM", "Outer SYRK", "Outer GEMM", "Panel GETRF",
        "Pivot propagation", "Inner pivot batch", "Inner TRSM", "Outer pivot batch",
        "Outer TRSM block", "Outer TRSM GEMM", "Outer TRSM direct"};
    return (stage >= 0 && stage < kNumStages) ? names[stage] : "unknown";
}

int hdbf_profile_num_stages(void) { return kNumStages; }

hdbf_status hdbf_profile_stages(hdbf_handle h, int max_stages, double* ms, double* flops,
                                int* calls)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    for (int st = 0; st < max_stages; ++st) {
        const bool in = st < kNumStages;
        if (ms) ms[st] = in ? h->stage_ms[st] : 0.0;
        if (flops) flops[st] = in ? h->stage_flops[st] : 0.0;
        if (calls) calls[st] = in ? h->stage_calls[st] : 0;
    }
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_set_panel_kernel(hdbf_handle h, int mode)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (mode < 0 || mode > 2) return HDBF_STATUS_INVALID_VALUE;
    if (mode != h->panel_mode) graph_cache_clear(h);
    h->panel_mode = mode;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_set_lookahead(hdbf_handle h, int enabled)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if ((enabled != 0) != (h->lookahead != 0)) graph_cache_clear(h);
    h->lookahead = enabled != 0;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_set_wait_limit(hdbf_handle h, unsigned int polls)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess ||
        cudaMemcpy(h->dev_small + kSmallSpin, &polls, sizeof(unsigned), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
        cudaGetLastError();
        return HDBF_STATUS_CUDA_ERROR;
    }
    h->spin_limit = polls;
    return HDBF_STATUS_SUCCESS;
}

hdbf_status hdbf_set_graph_mode(hdbf_handle h, int enabled)
{
    if (!h) return HDBF_STATUS_INVALID_HANDLE;
    h->use_graphs = enabled != 0;
    if (!h->use_graphs) graph_cache_clear(h);
    return HDBF_STATUS_SUCCESS;
}

}  // extern "C"
