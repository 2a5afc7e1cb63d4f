// chol_noalloc.cu -- variable-size Cholesky for callers that cannot allocate
// device memory (magma_dpotrf_vbatched_max_nocheck_noalloc).
//
// The regular entry point keeps its size-bucket lists in the queue's
// workspace, which is grown with cudaMalloc the first time a call needs more.
// Some callers cannot allow that: code that enqueues work while a CUDA graph is
// being captured (an allocation during capture breaks the capture), services
// that must fix every device allocation up front inside a memory budget, and
// code running inside an allocator's own callbacks. This variant instead uses
// a file-scope device array, g_chol_noalloc_scratch, sized for at most
// kNoAllocMaxBatch instances; it is part of the library image, so every GPU
// that loads the library holds it (about 2 MiB) until the process exits.
//
// Host code cannot pass the array's name to a kernel (on the host the name
// is only a stand-in, not a device address), so the first call on each device
// looks up the device address with cudaGetSymbolAddress, with that device
// current, and caches it. That first call should therefore happen before any
// stream capture. Every call reuses the same array, and its bucket counters
// are cleared at the start of each call; two calls whose work overlaps on the
// GPU (different streams, no ordering between them) would race on it, so
// callers must order them (for example by using one stream). The cached
// address belongs to the device's current context: after cudaDeviceReset (or
// anything else that destroys and recreates the primary context) the module is
// loaded again, possibly elsewhere, so a process that resets a device must not
// call this entry point on it afterwards. The size buckets run one after another
// on the queue's stream (the allocating entry point spreads them over auxiliary
// streams), so a batch of mixed sizes takes somewhat longer here.
#include "internal.h"
#include "chol_launch.h"
#include "vbatched.h"

#include <mutex>

namespace mb200 {

constexpr int kNoAllocMaxBatch = 65536;
constexpr int kNoAllocMaxDevices = 64;
constexpr size_t kNoAllocInts = 2 * kCholBuckets + (size_t)kCholBuckets * kNoAllocMaxBatch;

static __device__ __align__(256) int g_chol_noalloc_scratch[kNoAllocInts];

static int* g_scratch_addr[kNoAllocMaxDevices] = {};
static std::mutex g_scratch_mutex;

// Device address of g_chol_noalloc_scratch on `device` (looked up once, with
// that device current); nullptr if the lookup fails.
static int* noalloc_scratch(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices) {
        std::fprintf(stderr, "magma_dpotrf_vbatched_max_nocheck_noalloc: device %d is outside the %d devices "
                     "this entry point serves\n", device, kNoAllocMaxDevices);
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[device]) {
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e == cudaSuccess && prev != device) e = cudaSetDevice(device);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "magma_dpotrf_vbatched_max_nocheck_noalloc: cannot make device %d current: %s\n",
                         device, cudaGetErrorString(e));
            cudaGetLastError();
            return nullptr;
        }
        int* p = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_chol_noalloc_scratch);
        if (prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "libmagma_b200: cudaGetSymbolAddress(g_chol_noalloc_scratch) failed: %s\n",
                         cudaGetErrorString(e));
            cudaGetLastError();
            return nullptr;
        }
        g_scratch_addr[device] = p;
    }
    return g_scratch_addr[device];
}

}  // namespace mb200

using namespace mb200;

extern "C" magma_int_t magma_dpotrf_vbatched_max_nocheck_noalloc(magma_uplo_t uplo, magma_int_t* n,
                                                                  double** dA_array, magma_int_t* ldda,
                                                                  magma_int_t* info_array, magma_int_t batchCount,
                                                                  magma_int_t max_n, magma_queue_t queue) {
    if (batchCount > kNoAllocMaxBatch) {
        std::fprintf(stderr,
                     "magma_dpotrf_vbatched_max_nocheck_noalloc: batchCount %d exceeds the %d instances its "
                     "static scratch holds; split the batch or use magma_dpotrf_vbatched_max_nocheck\n",
                     (int)batchCount, kNoAllocMaxBatch);
        return -6;
    }
    if (batchCount <= 0 || max_n <= 0) return 0;
    const int top = chol_bucket_of(max_n);
    if (top < 0) return MAGMA_ERR_NOT_SUPPORTED;
    int* ws = noalloc_scratch(queue->device);
    if (!ws) return MAGMA_ERR_UNKNOWN;
    cudaMemsetAsync(info_array, 0, sizeof(int) * batchCount, queue->stream);
    int *counts, *lists;   // bucketize clears the counters before filling the lists
    magma_int_t rc = bucketize(n, batchCount, kCholEdges, kCholBuckets, queue->stream, ws, &counts, &lists);
    if (rc) return rc;
    const LuSizes sz{0, 0, 0, 0, 0, n, n, ldda, nullptr, nullptr};
    for (int b = top; b >= 0; --b) {
        const WorkList wl{lists + (size_t)b * batchCount, counts + b, 0};
        chol_bucket<double>(b, wl, batchCount, true, sz, uplo == MagmaUpper, dA_array, nullptr, info_array, true,
                            false, 1, queue->stream);
    }
    return launch_status();
}
