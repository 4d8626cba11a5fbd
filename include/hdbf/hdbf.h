/*
 * Runtime API of the B200 dense-factorization library (libhdbf.so).
 *
 * The reference passes a rocBLAS handle (rocblas_handle, owning a HIP stream)
 * as the first argument of every entry point and aborts the process on any
 * error (include/utils/common/error_check.h:9-28).  Here the first argument is
 * an hdbf_handle that owns a CUDA stream, a device workspace arena and the
 * status of the last call.  Entry points never exit the process: the
 * reference-shaped void functions record their status in the handle
 * (hdbf_get_last_status), and the hdbf_* functions return it directly.
 *
 * All matrix pointers are DEVICE pointers, column-major, with LP64 int sizes,
 * exactly as in the reference.  All work is enqueued on the handle's stream;
 * no entry point synchronises the host unless documented.
 */
#pragma once

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hdbf_context* hdbf_handle;

/* Opaque pool of CUDA streams; stands in for the reference's StreamPool class
 * (include/utils/memory/stream_pool.h:11-20, stream_pool.cpp:4-27). */
typedef struct hdbf_stream_pool StreamPool;

typedef enum hdbf_status {
    HDBF_STATUS_SUCCESS = 0,
    HDBF_STATUS_INVALID_HANDLE = 1,
    HDBF_STATUS_INVALID_VALUE = 2,
    HDBF_STATUS_ALLOC_FAILED = 3,
    HDBF_STATUS_CUDA_ERROR = 4,
    HDBF_STATUS_NOT_SUPPORTED = 5,
    HDBF_STATUS_TIMEOUT = 6,         /* a bounded device-side wait gave up */
    HDBF_STATUS_WORKSPACE_TOO_SMALL = 7 /* growth needed while a stream capture is active */
} hdbf_status;

/* Handle lifecycle (replaces rocblas_create_handle / rocblas_destroy_handle). */
hdbf_status hdbf_create(hdbf_handle* handle);
hdbf_status hdbf_destroy(hdbf_handle handle);

/* Stream binding (replaces rocblas_set_stream / rocblas_get_stream).  The
 * stream is a cudaStream_t passed as void* so this header needs no CUDA
 * include; NULL selects the legacy default stream. */
hdbf_status hdbf_set_stream(hdbf_handle handle, void* stream);
hdbf_status hdbf_get_stream(hdbf_handle handle, void** stream);

/* Status of the last reference-shaped (void) call made on this handle. */
hdbf_status hdbf_get_last_status(hdbf_handle handle);
const char* hdbf_status_string(hdbf_status status);

/* Grow the handle's device workspace to at least `bytes` now, so that later
 * calls made under CUDA stream capture do not need to allocate. */
hdbf_status hdbf_reserve_workspace(hdbf_handle handle, size_t bytes);
/* Workspace the factorization routines need for order n (bytes). */
size_t hdbf_workspace_bytes_for(int n);

/* Synchronise the handle's stream, then read and clear the device-side error
 * word written by bounded waits (a timed-out grid barrier sets it).  Returns
 * HDBF_STATUS_TIMEOUT if any kernel gave up, else the CUDA status. */
hdbf_status hdbf_check_device_errors(hdbf_handle handle);

/* Poll limit of every bounded device-side wait on this handle (the grid-wide
 * barriers and exchanges of the GETRF panel, diagonal-block Cholesky and
 * wavefront-solve kernels, FP32 and FP64).  0 restores the default, 2^22 polls
 * (about half a second with back-off).  A wait that runs out records
 * HDBF_STATUS_TIMEOUT, which hdbf_check_device_errors returns once (it then
 * clears the error word and the exchange state, keeping this limit), and the
 * kernel returns without finishing the factorization.  Takes effect for the
 * next launch, recorded graphs included; synchronous, not for use during a
 * stream capture. */
hdbf_status hdbf_set_wait_limit(hdbf_handle handle, unsigned int polls);

/* Stream pool (replaces `new StreamPool(n)` / `delete pool`). */
hdbf_status hdbf_stream_pool_create(int num_streams, StreamPool** pool);
hdbf_status hdbf_stream_pool_destroy(StreamPool* pool);
int hdbf_stream_pool_size(const StreamPool* pool);

/* Counter-based U[lo,hi) FP32 generator, bit-identical to the host oracle:
 * x[i] = top24(splitmix64(seed*0x9E3779B97F4A7C15 + (offset+i+1)*0xD1B54A32D192ED03))
 *        / 2^23 - 1, then mapped affinely to [lo,hi) (lo=-1, hi=1 exact). */
hdbf_status hdbf_fill_uniform(hdbf_handle handle, float* x, size_t count,
                              unsigned long long seed, unsigned long long offset);

/* Number of kernels this library launched since the handle was created
 * (a host-side counter; used to report gpu_launches). */
unsigned long long hdbf_launch_count(hdbf_handle handle);

/* Whole-factorization CUDA graphs (default on).  When enabled, the first
 * call of a factorization entry point with a given argument tuple records its
 * kernel chain as a CUDA graph; later calls with identical arguments replay it
 * on the handle's stream.  Calls made while the caller is itself capturing the
 * stream are recorded into the caller's graph instead. */
hdbf_status hdbf_set_graph_mode(hdbf_handle handle, int enabled);

/* GETRF panel-leaf kernel: 0 = automatic (thread-block cluster when the
 * column block fits in one cluster's shared memory, otherwise the
 * grid-wide publish-and-poll kernel), 1 = always the grid-wide kernel,
 * 2 = cluster only (blocks that do not fit still take the grid-wide kernel).
 * Both produce identical pivots and factors.  A new handle starts in the mode
 * named by the environment variable HDBF_PANEL_KERNEL (0, 1 or 2), else 0.
 * The panel recursion stops at leaves of 128 columns (the grid-wide kernel
 * takes up to 128; the cluster kernel up to 32, so mode 2 recurses to 32);
 * HDBF_PANEL_LEAF (32, 64 or 128) sets a new handle's leaf width, and
 * HDBF_PANEL_ROWS (64..4096, default 256) the rows each CTA of the grid-wide
 * kernel aims to hold. */
hdbf_status hdbf_set_panel_kernel(hdbf_handle handle, int mode);

/* Look-ahead in the double-blocked GETRF entry points with batched pivoting
 * or without pivoting (default on; HDBF_LOOKAHEAD=0 turns a new handle's
 * off).  The outer TRSM of the next outer block runs whole; its outer GEMM
 * then runs in column chunks of the inner panel width on the handle's
 * stream, while the inner panels of that block are factored, each as soon as
 * its chunk is updated, on a high-priority internal stream that joins the
 * handle's stream again at the end of the block.  Row interchanges of the
 * block's panels reach each later inner panel, composed, just before its
 * inner update.  Pivots and factors are the same as without look-ahead.
 * double_blocked_getrf (immediate pivoting) always runs serially. */
hdbf_status hdbf_set_lookahead(hdbf_handle handle, int enabled);

/* Per-launch event profiling of this library's kernels on the handle's
 * stream.  Between begin and end every launch is bracketed by CUDA events;
 * end synchronises the stream and returns, per kernel class (see
 * hdbf_profile_class_name), the summed device time in ms, the summed
 * algorithmic flops and bytes, and the launch count. */
hdbf_status hdbf_profile_begin(hdbf_handle handle);
hdbf_status hdbf_profile_end(hdbf_handle handle, int max_classes, double* ms, double* flops,
                             double* bytes, unsigned long long* launches);
const char* hdbf_profile_class_name(int cls);
int hdbf_profile_num_classes(void);

/* Per-stage split of the last hdbf_profile_begin/end interval: for each stage
 * of the double-blocked drivers (index 1 .. hdbf_profile_num_stages()-1, named
 * by hdbf_profile_stage_name as the reference's stage profilers name them:
 * "POTRF", "TRSM", "Inner GEMM", "Outer SYRK", "Outer GEMM", "Panel GETRF",
 * "Pivot propagation", "Inner pivot batch", "Inner TRSM", "Outer pivot batch",
 * "Outer TRSM block", "Outer TRSM GEMM", "Outer TRSM direct"), the summed
 * device time of its launches in ms, their algorithmic flops, and the number
 * of times the driver entered the stage.  Index 0 collects launches outside
 * any stage and is not reported. */
int hdbf_profile_num_stages(void);
const char* hdbf_profile_stage_name(int stage);
hdbf_status hdbf_profile_stages(hdbf_handle handle, int max_stages, double* ms, double* flops,
                                int* calls);

#ifdef __cplusplus
}
#endif
