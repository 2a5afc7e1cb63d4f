// lu_queue.cuh -- variable-size LU (getrf, and gesv = getrf + getrs NoTrans) of orders
// up to 512 in ONE launch: a persistent kernel, one 512-thread block per SM, whose warps
// take instances from a single device-side queue, largest first. The scheme is the
// one-launch Cholesky's (chol_queue.cuh): the size buckets' lists read from the top
// bucket down, teams of 512 threads that split in two whenever the drawn instance needs
// fewer threads, named barriers per team, per-warp shares of the dynamic shared memory:
//   512 threads  256 < max(m,n) <= 512   blocked getrf (thread = row) + blocked getrs
//   256          128 <          <= 256
//   128           64 <          <= 128
//    64           32 <          <=  64
//    32                max(m,n) <=  32   register-resident getrf / gesv, 8/16/32 columns
// The blocked teams use column chunks of 128 (64 for 128 threads, 32 for 64) so that
// every team's shared memory fits its warps' shares; the chunk width only groups the
// trailing columns, each element's updates keep their order. All paths apply the
// unblocked dgetf2 operations in order, so factors, pivots, info and NoTrans solutions
// are the same bits as the per-bucket kernels' and the oracle's. Counterparts in the
// reference: src/zgetrf_batched.cpp:222-351 (a launch sequence per call) and
// magmablas/gemm_template_kernel_vbatched.cuh:53-54 (grids sized by the largest instance).
#pragma once

#include "blocked_lu.cuh"
#include "getrs_blocked.cuh"
#include "small_lu_kernels.cuh"
#include "lu_sizes.h"

namespace mb200 {

constexpr int kLuQueueThreads = 512;
constexpr int kLuQueueWarps = kLuQueueThreads / 32;
constexpr int kLuQueueBuckets = 7;   // buckets 0..6: max(m, n) <= 512

// Buckets top..0 of a bucketize() result as one list; *head counts the tickets drawn.
struct LuQueue {
    const int* counts;
    const int* lists;
    int batch;
    int top;
    int* head;
};

template <int S> struct LuQueueTeam {   // column chunk and prefetch group of a blocked team
    static constexpr int CW = S >= 256 ? 128 : S == 128 ? 64 : 32;
    static constexpr int CB = S == 256 ? 4 : 8;
};

template <size_t A, size_t B> struct LuMaxSz { static constexpr size_t v = A > B ? A : B; };

template <typename T, int R>
struct LuQueueShare {
    template <int S>
    static constexpr size_t per_warp() {
        constexpr size_t f = sizeof(BlockedLuShared<T, 32, S, LuQueueTeam<S>::CW, false>);
        constexpr size_t s = sizeof(BlockedRsShared<T, S, R>);
        return ((f > s ? f : s) + S / 32 - 1) / (S / 32);
    }
    static constexpr size_t raw =
        LuMaxSz<LuMaxSz<sizeof(SmallLuShared<T, 32, 1>), per_warp<64>()>::v,
                LuMaxSz<per_warp<128>(), LuMaxSz<per_warp<256>(), per_warp<512>()>::v>::v>::v;
    static constexpr size_t bytes = (raw + 15) / 16 * 16;
};

__device__ __forceinline__ int lu_queue_barrier_id(int S, int w0) {
    return S == 512 ? 0 : S == 256 ? 1 + (w0 >> 3) : S == 128 ? 3 + (w0 >> 2) : 7 + (w0 >> 1);
}

// One instance on a team of S >= 64 threads: blocked getrf, then (SOLVE) getrs NoTrans.
template <typename T, int S, bool SOLVE, int R>
__device__ __forceinline__ void lu_queue_blocked(int id, const LuSizes& sz, T** dA, int** ipiv_array, T** dB,
                                                 int* info_array, unsigned char* base, const WarpRangeTeam& team) {
    using TT = LuQueueTeam<S>;
    const int m = sz.get_m(id), n = sz.get_n(id), lda = sz.get_lda(id);
    int* ipiv = ipiv_array ? ipiv_array[id] : nullptr;   // null: LU without pivoting
    auto& sh = *reinterpret_cast<BlockedLuShared<T, 32, S, TT::CW, false>*>(base);
    int info = 0;
    blocked_getrf<T, 32, S, TT::CW, TT::CB, false>(dA[id], m, n, lda, ipiv, info, sh, team);
    if (team.tid() == 0) info_array[id] = info;
    team.sync();   // the solve's shared memory overlays the factorisation's
    if constexpr (SOLVE) {
        // MAGMA's gesv solves regardless of info (src/zgesv_batched.cpp:137-147)
        const int nrhs = sz.get_nrhs(id);
        if (nrhs > 0) {
            auto& rs = *reinterpret_cast<BlockedRsShared<T, S, R>*>(base);
            blocked_getrs<T, S, R>(false, dA[id], n, lda, ipiv, dB[id], nrhs, sz.get_ldb(id), rs, team);
        }
    }
}

// One instance with max(m, n) <= 32 on one warp, in registers.
template <typename T, int NC, bool SOLVE, int R>
__device__ __forceinline__ void lu_queue_small_nc(int id, const LuSizes& sz, T** dA, int** ipiv_array, T** dB,
                                                  int* info_array, unsigned char* base, int lane) {
    auto& sh = *reinterpret_cast<SmallLuShared<T, NC, 1>*>(base);
    if constexpr (SOLVE) gesv_small_instance<T, NC, 1, R>(id, sz, dA, ipiv_array, dB, info_array, lane, sh);
    else getrf_small_instance<T, NC, 1>(id, sz, dA, ipiv_array, info_array, lane, sh);
    __syncwarp();
}

template <typename T, bool SOLVE, int R>
__device__ __forceinline__ void lu_queue_small(int id, int key, const LuSizes& sz, T** dA, int** ipiv_array, T** dB,
                                               int* info_array, unsigned char* base, int lane) {
    if (key <= 8) lu_queue_small_nc<T, 8, SOLVE, R>(id, sz, dA, ipiv_array, dB, info_array, base, lane);
    else if (key <= 16) lu_queue_small_nc<T, 16, SOLVE, R>(id, sz, dA, ipiv_array, dB, info_array, base, lane);
    else lu_queue_small_nc<T, 32, SOLVE, R>(id, sz, dA, ipiv_array, dB, info_array, base, lane);
}

template <typename T, bool SOLVE, int R>
__global__ void __launch_bounds__(kLuQueueThreads, 1)
lu_queue_kernel(LuQueue q, LuSizes sz, T** dA, int** ipiv_array, T** dB, int* info_array) {
    extern __shared__ __align__(16) unsigned char lu_queue_smem[];
    __shared__ int drawn[kLuQueueWarps];
    __shared__ int first[kLuQueueBuckets], count[kLuQueueBuckets];
    constexpr size_t share = LuQueueShare<T, R>::bytes;
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
    auto key_of = [&](int id) { return max(sz.get_m(id), sz.get_n(id)); };
    // teams of 512 .. 64 threads: blocked kernels
    int S = kLuQueueThreads, w0 = 0, t = -1;
    while (S >= 64) {
        if (t < 0) {
            if (warp == w0 && lane == 0) drawn[w0] = atomicAdd(q.head, 1);
            BarSync{lu_queue_barrier_id(S, w0), S}();
            t = drawn[w0];
            BarSync{lu_queue_barrier_id(S, w0), S}();   // every thread has read the slot before the next draw
        }
        if (t >= total) return;
        const int id = instance_at(t);
        const int key = key_of(id);
        const int need = key <= 32 ? 32 : key <= 64 ? 64 : key <= 128 ? 128 : key <= 256 ? 256 : 512;
        if (need < S) {   // split: the lower half keeps ticket t, the upper half draws anew
            S >>= 1;
            if (warp >= w0 + S / 32) {
                w0 += S / 32;
                t = -1;
            }
            continue;
        }
        unsigned char* base = lu_queue_smem + (size_t)w0 * share;
        const WarpRangeTeam team{w0 * 32, lu_queue_barrier_id(S, w0), S};
        switch (S) {
            case 512: lu_queue_blocked<T, 512, SOLVE, R>(id, sz, dA, ipiv_array, dB, info_array, base, team); break;
            case 256: lu_queue_blocked<T, 256, SOLVE, R>(id, sz, dA, ipiv_array, dB, info_array, base, team); break;
            case 128: lu_queue_blocked<T, 128, SOLVE, R>(id, sz, dA, ipiv_array, dB, info_array, base, team); break;
            default: lu_queue_blocked<T, 64, SOLVE, R>(id, sz, dA, ipiv_array, dB, info_array, base, team); break;
        }
        t = -1;
    }
    // single warps (max(m, n) <= 32): registers; the ticket travels by shuffle
    unsigned char* base = lu_queue_smem + (size_t)warp * share;
    while (true) {
        if (t < 0) {
            int d = 0;
            if (lane == 0) d = atomicAdd(q.head, 1);
            t = __shfl_sync(0xffffffffu, d, 0);
        }
        if (t >= total) return;
        const int id = instance_at(t);
        lu_queue_small<T, SOLVE, R>(id, key_of(id), sz, dA, ipiv_array, dB, info_array, base, lane);
        t = -1;
    }
}

}  // namespace mb200
