// vbatched.cu -- shared machinery of the variable-size ("vbatched") entry points:
// argument checking, max-size reduction and size bucketing, all on the device.
//
// Reference counterparts: magmablas/vbatched_check.cu:17-100 (checker kernels +
// host sync), magmablas/vbatched_aux.cu:504-590 (magma_imax_size_*). Instead of
// sizing one grid by the largest instance (so that every block of a smaller
// instance exits early, gemm_template_kernel_vbatched.cuh:53-54), instances
// are counting-sorted into size buckets and each bucket's kernel walks only
// its own list.
#include "internal.h"
#include "vbatched.h"
#include <mutex>
#include <map>
#include <atomic>

namespace mb200 {

__global__ void bucketize_kernel(const int* __restrict__ key, const int* __restrict__ key2, int batch,
                                 BucketEdges edges, int* __restrict__ counts, int* __restrict__ lists) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    const int v = key2 ? ((key[i] <= 0 || key2[i] <= 0) ? 0 : max(key[i], key2[i])) : key[i];
    if (v <= 0) return;                       // empty instances need no work
    int b = 0;
    while (b < edges.n - 1 && v > edges.e[b]) ++b;
    const int slot = atomicAdd(&counts[b], 1);
    lists[(size_t)b * batch + slot] = i;
}

__global__ void reduce_sizes_kernel(const int* __restrict__ a, const int* __restrict__ b, const int* __restrict__ c,
                                    int batch, int* __restrict__ out) {
    // out[0..2] = max of a, b, c; out[3..5] = min of a, b, c
    int mx[3] = {0, 0, 0}, mn[3] = {INT_MAX, INT_MAX, INT_MAX};
    const int* src[3] = {a, b, c};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int t = 0; t < 3; ++t)
            if (src[t]) { mx[t] = max(mx[t], src[t][i]); mn[t] = min(mn[t], src[t][i]); }
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        for (int off = 16; off > 0; off >>= 1) {
            mx[t] = max(mx[t], __shfl_xor_sync(0xffffffffu, mx[t], off));
            mn[t] = min(mn[t], __shfl_xor_sync(0xffffffffu, mn[t], off));
        }
        if ((threadIdx.x & 31) == 0) { atomicMax(&out[t], mx[t]); atomicMin(&out[3 + t], mn[t]); }
    }
}

// min over i of (ld[i] - rows[i]): negative when some leading dimension is too
// small (the reference's checkers test ld < rows, vbatched_check.cu:38-40, :852)
__global__ void ld_slack_kernel(const int* __restrict__ rows, const int* __restrict__ ld, int batch,
                                int* __restrict__ out, int at_least) {
    int mn = INT_MAX;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x)
        mn = min(mn, ld[i] - max(at_least, rows[i]));
    for (int off = 16; off > 0; off >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, off));
    if ((threadIdx.x & 31) == 0) atomicMin(out, mn);
}

__global__ void init_ints_kernel(int* p, int n, int v0, int v1, int split) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (i < split) ? v0 : v1;
}

magma_int_t bucketize(const int* key, int batch, const int* edges_host, int nb, cudaStream_t s, int* ws,
                      int** counts_out, int** lists_out) {
    return bucketize2(key, nullptr, batch, edges_host, nb, s, ws, counts_out, lists_out);
}

magma_int_t bucketize2(const int* key, const int* key2, int batch, const int* edges_host, int nb, cudaStream_t s,
                       int* ws, int** counts_out, int** lists_out) {
    // ws layout: [counts nb (padded to 2*nb)][lists nb*batch]; the edges travel as a kernel argument
    if (nb > BucketEdges::kMax) return MAGMA_ERR_NOT_SUPPORTED;
    BucketEdges edges;
    edges.n = nb;
    for (int b = 0; b < nb; ++b) edges.e[b] = edges_host[b];
    int* d_counts = ws;
    int* d_lists = ws + 2 * nb;
    cudaMemsetAsync(d_counts, 0, sizeof(int) * 2 * nb, s);   // counts and the nb spare counters after them
    bucketize_kernel<<<ceildiv(batch, 256), 256, 0, s>>>(key, key2, batch, edges, d_counts, d_lists);
    *counts_out = d_counts;
    *lists_out = d_lists;
    return launch_status();
}

size_t bucketize_ws_ints(int batch, int nb) { return (size_t)2 * nb + (size_t)nb * batch; }

// One block per bucket: a counting sort of the bucket's list by key, descending.
constexpr int kSortBins = 1024;
__global__ void __launch_bounds__(1024)
bucket_sort_kernel(const int* __restrict__ key, const int* __restrict__ key2, int batch, BucketEdges edges,
                   const int* __restrict__ counts, int* __restrict__ lists, int* __restrict__ tmp) {
    __shared__ int hist[kSortBins];
    __shared__ int warp_sum[32];
    const int b = blockIdx.x, cnt = counts[b];
    if (cnt <= 1) return;
    const int lo = (b == 0) ? 1 : edges.e[b - 1] + 1;
    int* list = lists + (size_t)b * batch;
    int* out = tmp + (size_t)b * batch;
    for (int i = threadIdx.x; i < kSortBins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    auto bin_of = [&](int id) {
        const int v = key2 ? max(key[id], key2[id]) : key[id];
        return kSortBins - 1 - min(max(v - lo, 0), kSortBins - 1);   // largest keys first
    };
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) atomicAdd(&hist[bin_of(list[i])], 1);
    __syncthreads();
    // exclusive scan of the 1024 bins: one bin per thread, warp scans, then the warp totals
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    int v = hist[t], x = v;
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = warp_sum[lane];
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, off);
            if (lane >= off) s += y;
        }
        warp_sum[lane] = s;   // inclusive
    }
    __syncthreads();
    hist[t] = x - v + (w > 0 ? warp_sum[w - 1] : 0);   // exclusive start of bin t
    __syncthreads();
    for (int i = t; i < cnt; i += blockDim.x) {
        const int id = list[i];
        out[atomicAdd(&hist[bin_of(id)], 1)] = id;
    }
    __syncthreads();
    for (int i = t; i < cnt; i += blockDim.x) list[i] = out[i];
}

size_t bucket_sort_ws_ints(int batch, int nb) { return (size_t)nb * batch; }

magma_int_t sort_buckets_desc(const int* key, const int* key2, int batch, const int* edges_host, int nb,
                              cudaStream_t s, const int* counts, int* lists, int* tmp) {
    if (nb > BucketEdges::kMax) return MAGMA_ERR_NOT_SUPPORTED;
    BucketEdges edges;
    edges.n = nb;
    for (int b = 0; b < nb; ++b) edges.e[b] = edges_host[b];
    bucket_sort_kernel<<<nb, kSortBins, 0, s>>>(key, key2, batch, edges, counts, lists, tmp);
    return launch_status();
}

// Device reduction of up to three size arrays, copied back to the host
// (the reference does the same with magma_imax_size_* + getvector + sync).
magma_int_t reduce_sizes(const int* a, const int* b, const int* c, int batch, magma_queue_t queue, int out[6]) {
    int* d = static_cast<int*>(queue_workspace(queue, 64));
    if (!d) return MAGMA_ERR_DEVICE_ALLOC;
    init_ints_kernel<<<1, 32, 0, queue->stream>>>(d, 6, 0, INT_MAX, 3);
    reduce_sizes_kernel<<<min(ceildiv(batch, 256), 148), 256, 0, queue->stream>>>(a, b, c, batch, d);
    cudaMemcpyAsync(out, d, sizeof(int) * 6, cudaMemcpyDeviceToHost, queue->stream);
    cudaStreamSynchronize(queue->stream);
    return launch_status();
}

static magma_int_t ld_slack_impl(const int* rows, const int* ld, int batch, magma_queue_t queue, int* out,
                                 int at_least) {
    int* d = static_cast<int*>(queue_workspace(queue, 64));
    if (!d) return MAGMA_ERR_DEVICE_ALLOC;
    init_ints_kernel<<<1, 32, 0, queue->stream>>>(d, 1, INT_MAX, INT_MAX, 1);
    ld_slack_kernel<<<min(ceildiv(batch, 256), 148), 256, 0, queue->stream>>>(rows, ld, batch, d, at_least);
    cudaMemcpyAsync(out, d, sizeof(int), cudaMemcpyDeviceToHost, queue->stream);
    cudaStreamSynchronize(queue->stream);
    return launch_status();
}

magma_int_t ld_slack(const int* rows, const int* ld, int batch, magma_queue_t queue, int* out) {
    return ld_slack_impl(rows, ld, batch, queue, out, INT_MIN);
}

magma_int_t ld_slack1(const int* rows, const int* ld, int batch, magma_queue_t queue, int* out) {
    return ld_slack_impl(rows, ld, batch, queue, out, 1);
}

int device_sm_count() {
    constexpr int kMaxDev = 64;
    static std::atomic<int> sms[kMaxDev] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDev) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        return max(1, v);
    }
    int v = sms[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        v = max(1, v);
        sms[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

void ensure_dynamic_smem(const void* kernel, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    int& have = done[{kernel, dev}];
    if (have >= bytes) return;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess) have = bytes;
    else cudaGetLastError();   // the launch that follows reports the failure
}

int resident_blocks(const void* kernel, int threads, size_t smem) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    return max(1, per_sm) * device_sm_count();
}

}  // namespace mb200
