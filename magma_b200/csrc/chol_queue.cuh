// chol_queue.cuh -- variable-size Cholesky (potrf / potrs / posv) of orders up
// to 512 in ONE launch: a persistent kernel, one 512-thread block per SM, whose
// warps take instances from a single device-side queue, largest first.
//
// The queue is the size buckets' lists read from the top bucket down (each list
// already sorted by n descending), so the instance behind ticket t never needs
// more threads than the one behind ticket t-1. A block starts as one team of 16
// warps. A team that draws an instance needing fewer threads splits in two: the
// lower half keeps the instance, the upper half draws the next ticket. Teams
// therefore only ever split, down to single warps:
//   512 threads  256 < n <= 512   blocked potrf (thread = row) + blocked potrs
//   256          128 < n <= 256
//   128           64 < n <= 128
//    64           32 < n <=  64
//    32                n <=  32   register-resident potrf (+ fused potrs), 8/16/32 columns
// A team synchronises on its own named barrier (0 for 512 threads; 1-2 for 256;
// 3-6 for 128; 7-14 for 64) and owns the shared memory of its warps, shares
// [w0, w0 + S/32) of the dynamic shared memory. Single warps leave the team loop
// for a loop of their own (tickets by shuffle): keeping the two loops apart keeps
// the register-resident small path from spilling under the block's 128 registers.
//
// Each instance runs the same device functions, in the same thread-per-row
// layout, as the per-bucket kernels of chol_kernels.cu, so the results are the
// same bits. Counterparts in the reference: src/zpotrf_vbatched.cpp:146-204 (a
// launch sequence per size class) and magmablas/gemm_template_kernel_vbatched.cuh:53-54
// (grids sized by the largest instance, smaller instances' blocks exit early).
#pragma once

#include "chol.cuh"
#include "chol_launch.h"
#include "lu_sizes.h"

namespace mb200 {

constexpr int kQueueThreads = 512;
constexpr int kQueueWarps = kQueueThreads / 32;
constexpr int kQueueBuckets = 7;   // buckets 0..6: n <= 512

// Buckets top..0 of a bucketize() result as one list; *head counts the tickets
// drawn so far (zero before the launch).
struct CholQueue {
    const int* counts;   // per bucket
    const int* lists;    // bucket b's list at lists + b * batch
    int batch;
    int top;             // highest bucket read (<= 6)
    int* head;
};

template <size_t A, size_t B> struct MaxSz { static constexpr size_t v = A > B ? A : B; };

// Shared memory of one warp's share: the largest per-warp need over the team sizes.
template <typename T, int R>
struct QueueShare {
    template <int S>
    static constexpr size_t per_warp() {
        constexpr size_t f = sizeof(BlockedCholShared<T, 32, S, 64>), s = sizeof(BlockedCholRsShared<T, S, R>);
        return ((f > s ? f : s) + S / 32 - 1) / (S / 32);
    }
    static constexpr size_t raw =
        MaxSz<MaxSz<sizeof(CholShared<T, 32>), per_warp<64>()>::v,
              MaxSz<per_warp<128>(), MaxSz<per_warp<256>(), per_warp<512>()>::v>::v>::v;
    static constexpr size_t bytes = (raw + 15) / 16 * 16;
};

__device__ __forceinline__ int queue_team_barrier_id(int S, int w0) {
    return S == 512 ? 0 : S == 256 ? 1 + (w0 >> 3) : S == 128 ? 3 + (w0 >> 2) : 7 + (w0 >> 1);
}

__device__ __forceinline__ void queue_team_sync(int S, int w0) {
    if (S == 32) __syncwarp();
    else BarSync{queue_team_barrier_id(S, w0), S}();
}

// One instance on a team of S threads (S >= 64): blocked potrf, then potrs.
template <typename T, int S, bool FACTOR, bool SOLVE, int R>
__device__ __forceinline__ void queue_blocked(int id, const LuSizes& sz, bool upper, T** dA, T** dB, int* info,
                                              unsigned char* base, const WarpRangeTeam& team) {
    const int n = sz.get_n(id), lda = sz.get_lda(id);
    if constexpr (FACTOR) {
        auto& sh = *reinterpret_cast<BlockedCholShared<T, 32, S, 64>*>(base);
        // FP64 teams of 256 and 512 threads: the trailing updates on the tensor cores (the same
        // bits as the CUDA-core form, which the smaller teams keep: with them as well the
        // kernel spills heavily under its 128 registers)
        constexpr bool kDmma = std::is_same<T, double>::value && S >= 256;
        const int inf = blocked_potrf<T, 32, S, 64, 8, WarpRangeTeam, kDmma, false>(dA[id], n, lda, upper, sh, team);
        if (team.tid() == 0 && info) info[id] = inf;
        team.sync();   // the solve's shared memory overlays the factor's
    }
    if constexpr (SOLVE) {
        // MAGMA's posv solves regardless of info (src/zposv_batched.cpp:123-141)
        const int nrhs = sz.get_nrhs(id);
        if (nrhs > 0) {
            auto& rs = *reinterpret_cast<BlockedCholRsShared<T, S, R>*>(base);
            blocked_potrs<T, S, R>(dA[id], n, lda, upper, dB[id], nrhs, sz.get_ldb(id), rs, team);
        }
    }
}

// One instance with n <= 32 on one warp, in registers.
template <typename T, int NC, bool FACTOR, bool SOLVE, int R>
__device__ __forceinline__ void queue_small_nc(int id, const LuSizes& sz, bool upper, T** dA, T** dB, int* info,
                                               unsigned char* base, int lane) {
    auto& sh = *reinterpret_cast<CholShared<T, NC>*>(base);
    if constexpr (FACTOR) chol_small_instance<T, NC, 1, R, SOLVE>(id, sz, upper, dA, dB, info, lane, sh);
    else potrs_small_instance<T, NC, 1, R>(id, sz, upper, dA, dB, lane, sh);
    __syncwarp();
}

template <typename T, bool FACTOR, bool SOLVE, int R>
__device__ __forceinline__ void queue_small(int id, int n, const LuSizes& sz, bool upper, T** dA, T** dB, int* info,
                                            unsigned char* base, int lane) {
    if (n <= 8) queue_small_nc<T, 8, FACTOR, SOLVE, R>(id, sz, upper, dA, dB, info, base, lane);
    else if (n <= 16) queue_small_nc<T, 16, FACTOR, SOLVE, R>(id, sz, upper, dA, dB, info, base, lane);
    else queue_small_nc<T, 32, FACTOR, SOLVE, R>(id, sz, upper, dA, dB, info, base, lane);
}

template <typename T, bool FACTOR, bool SOLVE, int R>
__global__ void __launch_bounds__(kQueueThreads, 1)
chol_queue_kernel(CholQueue q, LuSizes sz, bool upper, T** dA, T** dB, int* info) {
    extern __shared__ __align__(16) unsigned char queue_smem[];
    __shared__ int drawn[kQueueWarps];
    __shared__ int first[kQueueBuckets], count[kQueueBuckets];
    constexpr size_t share = QueueShare<T, R>::bytes;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        int t = 0;
        for (int b = q.top; b >= 0; --b) {
            first[b] = t;
            count[b] = q.counts[b];
            t += count[b];
        }
    }
    __syncthreads();
    const int total = first[0] + count[0];
    auto instance_at = [&](int t) {
        int b = q.top;   // bucket b holds tickets [first[b], first[b] + count[b])
        while (b > 0 && t >= first[b] + count[b]) --b;
        return q.lists[(size_t)b * q.batch + (t - first[b])];
    };
    // teams of 512 .. 64 threads: blocked kernels
    int S = kQueueThreads, w0 = 0, t = -1;
    while (S >= 64) {
        if (t < 0) {
            if (warp == w0 && lane == 0) drawn[w0] = atomicAdd(q.head, 1);
            queue_team_sync(S, w0);
            t = drawn[w0];
            queue_team_sync(S, w0);   // every thread has read the slot before the next draw
        }
        if (t >= total) return;
        const int id = instance_at(t);
        const int n = sz.get_n(id);
        const int need = n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512;
        if (need < S) {   // split: the lower half keeps ticket t, the upper half draws anew
            S >>= 1;
            if (warp >= w0 + S / 32) {
                w0 += S / 32;
                t = -1;
            }
            continue;
        }
        unsigned char* base = queue_smem + (size_t)w0 * share;
        const WarpRangeTeam team{w0 * 32, queue_team_barrier_id(S, w0), S};
        switch (S) {
            case 512: queue_blocked<T, 512, FACTOR, SOLVE, R>(id, sz, upper, dA, dB, info, base, team); break;
            case 256: queue_blocked<T, 256, FACTOR, SOLVE, R>(id, sz, upper, dA, dB, info, base, team); break;
            case 128: queue_blocked<T, 128, FACTOR, SOLVE, R>(id, sz, upper, dA, dB, info, base, team); break;
            default: queue_blocked<T, 64, FACTOR, SOLVE, R>(id, sz, upper, dA, dB, info, base, team); break;
        }
        t = -1;
    }
    // single warps (n <= 32): registers; the ticket travels by shuffle
    unsigned char* base = queue_smem + (size_t)warp * share;
    while (true) {
        if (t < 0) {
            int d = 0;
            if (lane == 0) d = atomicAdd(q.head, 1);
            t = __shfl_sync(0xffffffffu, d, 0);
        }
        if (t >= total) return;
        const int id = instance_at(t);
        queue_small<T, FACTOR, SOLVE, R>(id, sz.get_n(id), sz, upper, dA, dB, info, base, lane);
        t = -1;
    }
}

}  // namespace mb200
