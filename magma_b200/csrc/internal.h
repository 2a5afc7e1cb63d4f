// internal.h -- private runtime state shared by the host side of libmagma_b200.
//
// The queue mirrors the role of MAGMA's struct magma_queue
// (control/magma_internal.h:86-139): a device id plus the CUDA stream all work
// is enqueued on. Unlike the reference it also owns a grow-only device
// workspace, so batched routines never call cudaMalloc on their call path
// (the reference mallocs and frees ~20 buffers per call,
// src/zgetrf_batched.cpp:148-194 and :356-376).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdio>
#include "../../include/magma_b200.h"

struct magma_queue {
    int          device;
    cudaStream_t stream;
    bool         own_stream;
    // grow-only workspace owned by the queue, never larger than ws_limit
    void*        ws;
    size_t       ws_bytes;
    size_t       ws_limit;
    // host-pinned staging word used by routines that must read one value back
    int*         h_flag;
    // auxiliary streams for independent work (size buckets), created on first use
    cudaStream_t aux[4];
    cudaEvent_t  ev_fork;
    cudaEvent_t  ev_join[4];
    bool         aux_ready;
    // optional stage timing (magma_b200_stage_timing): events at stage boundaries
    bool         stage_on;
    int          stage_n;
    cudaEvent_t  stage_ev[8];
};

namespace mb200 {

// Returns a device workspace of at least `bytes` on `queue`, growing it when
// needed. Growing synchronises the queue's stream (the old buffer may still be
// in use by enqueued work) -- callers that capture CUDA graphs reserve the
// workspace once before capture with magma_queue_reserve_workspace(). Returns
// nullptr when the allocation fails or `bytes` exceeds the queue's limit
// (magma_b200_queue_set_workspace_limit); callers report MAGMA_ERR_DEVICE_ALLOC.
void* queue_workspace(magma_queue_t queue, size_t bytes);

// Fork/join of the queue's auxiliary streams: queue_fork makes every auxiliary
// stream wait for the work enqueued so far on the queue's stream, queue_aux(i)
// names one, and queue_join makes the queue's stream wait for all of them. Work
// that is independent (one size bucket per auxiliary stream) then runs
// concurrently, inside CUDA-graph capture too (the fork and join are event
// edges). The streams are created on the first fork, which therefore has to
// happen outside capture (the eager call that also sizes the workspace).
constexpr int kAuxStreams = 4;
magma_int_t queue_fork(magma_queue_t queue);
inline cudaStream_t queue_aux(magma_queue_t queue, int i) { return queue->aux[i % kAuxStreams]; }
void queue_join(magma_queue_t queue);

// Stage timing: when enabled on the queue, multi-kernel routines record an event
// on the queue's stream before their first stage and after each stage.
void queue_stage_begin(magma_queue_t queue);
void queue_stage_mark(magma_queue_t queue);

// Records a CUDA launch error as a MAGMA error code (0 when none).
inline magma_int_t launch_status() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "libmagma_b200: CUDA launch failed: %s\n", cudaGetErrorString(e));
        return MAGMA_ERR_UNKNOWN;
    }
    return MAGMA_SUCCESS;
}

inline int ceildiv(long a, long b) { return (int)((a + b - 1) / b); }

// SM count of the current device (looked up once per device).
int device_sm_count();

// Raises `kernel`'s dynamic shared-memory limit on the current device to at least
// `bytes`, calling cudaFuncSetAttribute only the first time per (kernel, device, size).
void ensure_dynamic_smem(const void* kernel, int bytes);

}  // namespace mb200
