// runtime.cu -- MAGMA runtime entry points (init, queues, memory, copies,
// error reporting, pointer-array helpers).
//
// Behaviour follows the reference routines cited beside each function; the
// implementation is the library's own (no cuBLAS/cuSPARSE handles are
// created: the batched path does not use them).
#include "internal.h"
#include <algorithm>

#include <atomic>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace {
std::mutex g_init_mutex;
int g_init_count = 0;
}  // namespace

extern "C" {

// interface_cuda/interface.cpp:168 -- reference-counted initialisation.
magma_int_t magma_init(void) {
    std::lock_guard<std::mutex> lock(g_init_mutex);
    if (g_init_count == 0) {
        int ndev = 0;
        cudaError_t e = cudaGetDeviceCount(&ndev);
        if (e != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            return MAGMA_ERR_UNKNOWN;
        }
    }
    ++g_init_count;
    return MAGMA_SUCCESS;
}

// interface_cuda/interface.cpp:246
magma_int_t magma_finalize(void) {
    std::lock_guard<std::mutex> lock(g_init_mutex);
    if (g_init_count <= 0) return MAGMA_ERR_NOT_INITIALIZED;
    --g_init_count;
    return MAGMA_SUCCESS;
}

// interface_cuda/error.cpp:112 -- message text for the codes this library returns.
const char* magma_strerror(magma_int_t err) {
    switch (err) {
        case MAGMA_SUCCESS:             return "success";
        case MAGMA_ERR:                 return "unknown error";
        case MAGMA_ERR_NOT_INITIALIZED: return "not initialized";
        case MAGMA_ERR_NOT_SUPPORTED:   return "not supported";
        case MAGMA_ERR_ILLEGAL_VALUE:   return "illegal value";
        case MAGMA_ERR_HOST_ALLOC:      return "cannot allocate memory on CPU host";
        case MAGMA_ERR_DEVICE_ALLOC:    return "cannot allocate memory on GPU device";
        case MAGMA_ERR_INVALID_PTR:     return "invalid pointer";
        case MAGMA_ERR_UNKNOWN:         return "unknown error";
        case MAGMA_ERR_NOT_IMPLEMENTED: return "not implemented";
        case MAGMA_ERR_NAN:             return "NaN detected";
        default:
            if (err < 0 && err > MAGMA_ERR) return "function-specific error, see documentation";
            return "unknown MAGMA error code";
    }
}

// control/xerbla.cpp:51 -- same four message forms as the reference.
void magma_xerbla(const char* srname, magma_int_t neg_info) {
    if (neg_info < 0) {
        std::fprintf(stderr, "Error in %s, function-specific error (info = %lld)\n",
                     srname, (long long)-neg_info);
    } else if (neg_info == 0) {
        std::fprintf(stderr, "No error, why is %s calling xerbla? (info = %lld)\n",
                     srname, (long long)-neg_info);
    } else if (neg_info >= -MAGMA_ERR) {
        std::fprintf(stderr, "Error in %s, %s (info = %lld)\n",
                     srname, magma_strerror(-neg_info), (long long)-neg_info);
    } else {
        std::fprintf(stderr, "On entry to %s, parameter %lld had an illegal value (info = %lld)\n",
                     srname, (long long)neg_info, (long long)-neg_info);
    }
}

void magma_getdevice(magma_device_t* dev) {
    int d = 0;
    cudaGetDevice(&d);
    *dev = d;
}

void magma_setdevice(magma_device_t dev) { cudaSetDevice(dev); }

// interface_cuda/alloc.cpp:60 -- zero-byte requests allocate one byte, as the reference.
magma_int_t magma_malloc(magma_ptr* ptr_ptr, size_t bytes) {
    if (bytes == 0) bytes = 1;
    if (cudaMalloc(ptr_ptr, bytes) != cudaSuccess) {
        cudaGetLastError();
        *ptr_ptr = nullptr;
        return MAGMA_ERR_DEVICE_ALLOC;
    }
    return MAGMA_SUCCESS;
}

// interface_cuda/alloc.cpp:93
magma_int_t magma_free_internal(magma_ptr ptr, const char* func, const char* file, int line) {
    cudaError_t e = cudaFree(ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        std::fprintf(stderr, "magma_free: %s at %s:%d in %s\n", cudaGetErrorString(e), file, line, func);
        return MAGMA_ERR_INVALID_PTR;
    }
    return MAGMA_SUCCESS;
}

// interface_cuda/alloc.cpp:242 -- page-locked host memory (portable across contexts);
// zero-byte requests allocate a minimal block, as the reference.
magma_int_t magma_malloc_pinned(void** ptr_ptr, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (cudaHostAlloc(ptr_ptr, bytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        *ptr_ptr = nullptr;
        return MAGMA_ERR_HOST_ALLOC;
    }
    return MAGMA_SUCCESS;
}

// interface_cuda/alloc.cpp:276
magma_int_t magma_free_pinned_internal(void* ptr, const char* func, const char* file, int line) {
    cudaError_t e = cudaFreeHost(ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        std::fprintf(stderr, "magma_free_pinned: %s at %s:%d in %s\n", cudaGetErrorString(e), file, line, func);
        return MAGMA_ERR_INVALID_PTR;
    }
    return MAGMA_SUCCESS;
}

// interface_cuda/interface.cpp:690 -- a queue with its own (non-blocking) stream.
void magma_queue_create_internal(magma_device_t device, magma_queue_t* queue_ptr,
                                 const char*, const char*, int) {
    magma_queue* q = new magma_queue();
    q->device = device;
    q->own_stream = true;
    q->ws = nullptr;
    q->ws_bytes = 0;
    q->ws_limit = SIZE_MAX;
    q->h_flag = nullptr;
    q->aux_ready = false;
    q->stage_on = false;
    q->stage_n = 0;
    cudaSetDevice(device);
    cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking);
    *queue_ptr = q;
}

// interface_cuda/interface.cpp:763 -- wrap a caller's stream; the handles are
// accepted for ABI compatibility and not used.
void magma_queue_create_from_cuda_internal(magma_device_t device, cudaStream_t stream,
                                           cublasHandle_t, cusparseHandle_t,
                                           magma_queue_t* queue_ptr,
                                           const char*, const char*, int) {
    magma_queue* q = new magma_queue();
    q->device = device;
    q->own_stream = false;
    q->stream = stream;
    q->ws = nullptr;
    q->ws_bytes = 0;
    q->ws_limit = SIZE_MAX;
    q->h_flag = nullptr;
    q->aux_ready = false;
    q->stage_on = false;
    q->stage_n = 0;
    *queue_ptr = q;
}

void magma_queue_destroy_internal(magma_queue_t queue, const char*, const char*, int) {
    if (!queue) return;
    cudaStreamSynchronize(queue->stream);
    if (queue->ws) cudaFree(queue->ws);
    if (queue->h_flag) cudaFreeHost(queue->h_flag);
    if (queue->aux_ready) {
        for (int i = 0; i < mb200::kAuxStreams; ++i) {
            cudaStreamSynchronize(queue->aux[i]);
            cudaStreamDestroy(queue->aux[i]);
            cudaEventDestroy(queue->ev_join[i]);
        }
        cudaEventDestroy(queue->ev_fork);
    }
    if (queue->stage_on)
        for (int i = 0; i < 8; ++i) cudaEventDestroy(queue->stage_ev[i]);
    if (queue->own_stream) cudaStreamDestroy(queue->stream);
    delete queue;
}

// interface_cuda/interface.cpp:871
void magma_queue_sync_internal(magma_queue_t queue, const char* func, const char* file, int line) {
    cudaError_t e = cudaStreamSynchronize(queue ? queue->stream : nullptr);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "CUDA runtime error: %s in %s at %s:%d\n",
                     cudaGetErrorString(e), func, file, line);
    }
}

magma_int_t magma_queue_get_device(magma_queue_t queue) { return queue->device; }
cudaStream_t magma_queue_get_cuda_stream(magma_queue_t queue) { return queue->stream; }

// Reserves at least `bytes` of queue workspace ahead of time so that later
// calls (for example inside CUDA graph capture) never allocate.
magma_int_t magma_queue_reserve_workspace(magma_queue_t queue, size_t bytes) {
    return mb200::queue_workspace(queue, bytes) ? MAGMA_SUCCESS : MAGMA_ERR_DEVICE_ALLOC;
}

// include/magma_copy.h:45-84 -- strided vector copies.
static void copy_vector(magma_int_t n, magma_int_t es, const void* src, magma_int_t incs,
                        void* dst, magma_int_t incd, cudaMemcpyKind kind, magma_queue_t queue,
                        bool sync) {
    if (n <= 0) return;
    cudaStream_t s = queue ? queue->stream : nullptr;
    if (incs == 1 && incd == 1) {
        cudaMemcpyAsync(dst, src, (size_t)n * es, kind, s);
    } else {
        cudaMemcpy2DAsync(dst, (size_t)incd * es, src, (size_t)incs * es, es, n, kind, s);
    }
    if (sync) cudaStreamSynchronize(s);
}

void magma_setvector_internal(magma_int_t n, magma_int_t es, const void* hx, magma_int_t incx,
                              magma_ptr dy, magma_int_t incy, magma_queue_t queue,
                              const char*, const char*, int) {
    copy_vector(n, es, hx, incx, dy, incy, cudaMemcpyHostToDevice, queue, true);
}
void magma_getvector_internal(magma_int_t n, magma_int_t es, const void* dx, magma_int_t incx,
                              void* hy, magma_int_t incy, magma_queue_t queue,
                              const char*, const char*, int) {
    copy_vector(n, es, dx, incx, hy, incy, cudaMemcpyDeviceToHost, queue, true);
}
void magma_setvector_async_internal(magma_int_t n, magma_int_t es, const void* hx, magma_int_t incx,
                                    magma_ptr dy, magma_int_t incy, magma_queue_t queue,
                                    const char*, const char*, int) {
    copy_vector(n, es, hx, incx, dy, incy, cudaMemcpyHostToDevice, queue, false);
}
void magma_getvector_async_internal(magma_int_t n, magma_int_t es, const void* dx, magma_int_t incx,
                                    void* hy, magma_int_t incy, magma_queue_t queue,
                                    const char*, const char*, int) {
    copy_vector(n, es, dx, incx, hy, incy, cudaMemcpyDeviceToHost, queue, false);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Pointer-array builders (magmablas/zset_pointer.cu:17-26, set_pointer.cu:72).
// The reference launches one 1-thread block per instance; here one thread
// writes one pointer and a 256-thread block covers 256 instances.
template <typename T>
__global__ void set_pointer_kernel(T** out, T* in, long lda, long row, long col, long offset, int batch) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < batch) out[i] = in + (long)i * offset + row + col * lda;
}

template <typename T>
static void set_pointer(T** out, T* in, magma_int_t lda, magma_int_t row, magma_int_t col,
                        magma_int_t offset, magma_int_t batch, magma_queue_t queue) {
    if (batch <= 0) return;
    set_pointer_kernel<T><<<mb200::ceildiv(batch, 256), 256, 0, queue->stream>>>(
        out, in, lda, row, col, offset, batch);
}

extern "C" {
void magma_dset_pointer(double** out, double* in, magma_int_t lda, magma_int_t row, magma_int_t col,
                        magma_int_t off, magma_int_t batch, magma_queue_t queue) {
    set_pointer(out, in, lda, row, col, off, batch, queue);
}
void magma_sset_pointer(float** out, float* in, magma_int_t lda, magma_int_t row, magma_int_t col,
                        magma_int_t off, magma_int_t batch, magma_queue_t queue) {
    set_pointer(out, in, lda, row, col, off, batch, queue);
}
void magma_iset_pointer(magma_int_t** out, magma_int_t* in, magma_int_t lda, magma_int_t row,
                        magma_int_t col, magma_int_t off, magma_int_t batch, magma_queue_t queue) {
    set_pointer(out, in, lda, row, col, off, batch, queue);
}
}  // extern "C"

// Every queue owns a stream and 4 auxiliary streams, so a process with a few queues
// (the request loop runs 4: 20 streams) exceeds the driver's default of 8 hardware
// work queues, and streams that share one are serialised: a small request's kernel
// waited behind another class's 18 ms factorisation (measured: small-request p50
// 3-7 ms instead of 0.1-0.5 ms under mixed load). When the library is loaded before
// the process creates its CUDA context (any program linked against it), this asks the
// driver for 32 hardware queues; a value the caller already set is kept, and a context
// that already exists is not affected.
__attribute__((constructor)) static void mb200_request_hw_queues() {
    setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
}

namespace mb200 {
magma_int_t queue_fork(magma_queue_t queue) {
    if (!queue->aux_ready) {
        bool ok = cudaEventCreateWithFlags(&queue->ev_fork, cudaEventDisableTiming) == cudaSuccess;
        for (int i = 0; i < kAuxStreams && ok; ++i)
            ok = cudaStreamCreateWithFlags(&queue->aux[i], cudaStreamNonBlocking) == cudaSuccess &&
                 cudaEventCreateWithFlags(&queue->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            return MAGMA_ERR_UNKNOWN;
        }
        queue->aux_ready = true;
    }
    cudaEventRecord(queue->ev_fork, queue->stream);
    for (int i = 0; i < kAuxStreams; ++i) cudaStreamWaitEvent(queue->aux[i], queue->ev_fork, 0);
    return MAGMA_SUCCESS;
}

void queue_stage_begin(magma_queue_t queue) {
    if (!queue->stage_on) return;
    queue->stage_n = 0;
    queue_stage_mark(queue);
}

void queue_stage_mark(magma_queue_t queue) {
    if (!queue->stage_on || queue->stage_n >= 8) return;
    cudaEventRecord(queue->stage_ev[queue->stage_n++], queue->stream);
}

void queue_join(magma_queue_t queue) {
    for (int i = 0; i < kAuxStreams; ++i) {
        cudaEventRecord(queue->ev_join[i], queue->aux[i]);
        cudaStreamWaitEvent(queue->stream, queue->ev_join[i], 0);
    }
}

void* queue_workspace(magma_queue_t queue, size_t bytes) {
    if (bytes <= queue->ws_bytes) return queue->ws;
    if (bytes > queue->ws_limit) return nullptr;
    // round up to 2 MiB so that small growth steps do not reallocate (within the limit)
    size_t want = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    want = std::min(want, queue->ws_limit);
    if (queue->ws) {
        cudaStreamSynchronize(queue->stream);
        cudaFree(queue->ws);
        queue->ws = nullptr;
        queue->ws_bytes = 0;
    }
    void* p = nullptr;
    if (cudaMalloc(&p, want) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    queue->ws = p;
    queue->ws_bytes = want;
    return p;
}
}  // namespace mb200

extern "C" {

magma_int_t magma_b200_queue_set_workspace_limit(magma_queue_t queue, size_t bytes) {
    if (!queue) return -1;
    queue->ws_limit = bytes;
    if (queue->ws_bytes > bytes) {   // the queue holds no more than its limit from here on
        cudaStreamSynchronize(queue->stream);
        cudaFree(queue->ws);
        queue->ws = nullptr;
        queue->ws_bytes = 0;
    }
    return MAGMA_SUCCESS;
}

magma_int_t magma_b200_stage_timing(magma_queue_t queue, magma_int_t enable) {
    if (!queue) return -1;
    if (enable && !queue->stage_on) {
        for (int i = 0; i < 8; ++i)
            if (cudaEventCreate(&queue->stage_ev[i]) != cudaSuccess) {
                cudaGetLastError();
                return MAGMA_ERR_UNKNOWN;
            }
        queue->stage_on = true;
    } else if (!enable && queue->stage_on) {
        cudaStreamSynchronize(queue->stream);
        for (int i = 0; i < 8; ++i) cudaEventDestroy(queue->stage_ev[i]);
        queue->stage_on = false;
    }
    queue->stage_n = 0;
    return MAGMA_SUCCESS;
}

magma_int_t magma_b200_stage_times(magma_queue_t queue, float* ms, magma_int_t max) {
    if (!queue) return -1;
    if (!queue->stage_on || queue->stage_n < 2) return 0;
    const int k = std::min<int>(max, queue->stage_n - 1);
    cudaEventSynchronize(queue->stage_ev[queue->stage_n - 1]);
    for (int i = 0; i < k; ++i) cudaEventElapsedTime(&ms[i], queue->stage_ev[i], queue->stage_ev[i + 1]);
    return k;
}

}  // extern "C"
