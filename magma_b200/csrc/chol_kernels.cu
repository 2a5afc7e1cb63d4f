// chol_kernels.cu -- batched Cholesky kernels (fixed and variable size) and
// their host launchers. Device code in chol.cuh.
#include "internal.h"
#include "chol.cuh"
#include "lu_sizes.h"
#include "vbatched.h"
#include "chol_launch.h"

namespace mb200 {

template <int NW> struct CholShape { static constexpr int MPB = (NW == 1) ? 4 : 1; };

// ---- register-resident potrf (+ optional fused potrs), thread = row ----
template <typename T, int NC, int NW, int R, bool SOLVE>
__global__ void __launch_bounds__(32 * NW * CholShape<NW>::MPB)
chol_small_kernel(WorkList wl, LuSizes sz, bool upper, T** dA_array, T** dB_array, int* info_array) {
    constexpr int MPB = CholShape<NW>::MPB;
    __shared__ CholShared<T, NC> shm[MPB];
    const int local = (NW == 1) ? (threadIdx.x >> 5) : 0;
    const int tid = (NW == 1) ? (threadIdx.x & 31) : threadIdx.x;
    for (int w = blockIdx.x * MPB + local; w < wl.size(); w += gridDim.x * MPB) {
        chol_small_instance<T, NC, NW, R, SOLVE>(wl.at(w), sz, upper, dA_array, dB_array, info_array, tid,
                                                 shm[local]);
        mat_sync<NW>();
    }
}

// ---- register-resident potrs only ----
template <typename T, int NC, int NW, int R>
__global__ void __launch_bounds__(32 * NW * CholShape<NW>::MPB)
potrs_small_kernel(WorkList wl, LuSizes sz, bool upper, T** dA_array, T** dB_array) {
    constexpr int MPB = CholShape<NW>::MPB;
    __shared__ CholShared<T, NC> shm[MPB];
    const int local = (NW == 1) ? (threadIdx.x >> 5) : 0;
    const int tid = (NW == 1) ? (threadIdx.x & 31) : threadIdx.x;
    for (int w = blockIdx.x * MPB + local; w < wl.size(); w += gridDim.x * MPB) {
        potrs_small_instance<T, NC, NW, R>(wl.at(w), sz, upper, dA_array, dB_array, tid, shm[local]);
        mat_sync<NW>();
    }
}

// ---- blocked potrf / potrs, one matrix per block ----
template <typename T, int NB, int NT, int CW, int CB>
__global__ void __launch_bounds__(NT, (NT <= 128 ? 4 : NT == 256 ? 2 : 1))
potrf_blocked_kernel(WorkList wl, LuSizes sz, bool upper, T** dA_array, int* info_array) {
    extern __shared__ __align__(16) unsigned char potrf_smem[];
    BlockedCholShared<T, NB, NT, CW>& sh = *reinterpret_cast<BlockedCholShared<T, NB, NT, CW>*>(potrf_smem);
    for (int w = blockIdx.x; w < wl.size(); w += gridDim.x) {
        const int id = wl.at(w);
        const int n = sz.get_n(id), lda = sz.get_lda(id);
        int info = 0;
        // FP64: the trailing updates on the tensor cores (the same bits as the CUDA-core form)
        if (n > 0) info = blocked_potrf<T, NB, NT, CW, CB, BlockTeam, std::is_same<T, double>::value>(
                       dA_array[id], n, lda, upper, sh);
        if (threadIdx.x == 0 && info_array) info_array[id] = info;
        __syncthreads();
    }
}

template <typename T, int NT, int R>
__global__ void __launch_bounds__(NT)
potrs_blocked_kernel(WorkList wl, LuSizes sz, bool upper, T** dA_array, T** dB_array) {
    __shared__ BlockedCholRsShared<T, NT, R> sh;
    for (int w = blockIdx.x; w < wl.size(); w += gridDim.x) {
        const int id = wl.at(w);
        const int n = sz.get_n(id), lda = sz.get_lda(id), nrhs = sz.get_nrhs(id), ldb = sz.get_ldb(id);
        if (n > 0 && nrhs > 0) blocked_potrs<T, NT, R>(dA_array[id], n, lda, upper, dB_array[id], nrhs, ldb, sh);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Launchers. Each bucket launcher covers instances with n in (lo, hi].
template <typename K>
static int grid_for(K kernel, int threads, int items_upper_bound, bool bounded, size_t smem = 0) {
    if (!bounded) return max(1, items_upper_bound);
    const int res = resident_blocks((const void*)kernel, threads, smem);
    return max(1, min(items_upper_bound, res));
}

template <typename T, int NC, int NW>
static void launch_chol_small(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, bool upper,
                              T** A, T** B, int* info, bool solve, int max_nrhs, cudaStream_t s) {
    constexpr int MPB = CholShape<NW>::MPB;
    const int threads = 32 * NW * MPB;
    const int items = ceildiv(bound, MPB);
    if (!solve) {
        auto k = chol_small_kernel<T, NC, NW, 1, false>;
        k<<<grid_for(k, threads, items, persistent), threads, 0, s>>>(wl, sz, upper, A, B, info);
    } else if (max_nrhs <= 1) {
        auto k = chol_small_kernel<T, NC, NW, 1, true>;
        k<<<grid_for(k, threads, items, persistent), threads, 0, s>>>(wl, sz, upper, A, B, info);
    } else if (max_nrhs <= 4) {
        auto k = chol_small_kernel<T, NC, NW, 4, true>;
        k<<<grid_for(k, threads, items, persistent), threads, 0, s>>>(wl, sz, upper, A, B, info);
    } else {
        auto k = chol_small_kernel<T, NC, NW, 8, true>;
        k<<<grid_for(k, threads, items, persistent), threads, 0, s>>>(wl, sz, upper, A, B, info);
    }
}

template <typename T, int NC, int NW>
static void launch_potrs_small(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, bool upper,
                               T** A, T** B, int max_nrhs, cudaStream_t s) {
    constexpr int MPB = CholShape<NW>::MPB;
    const int threads = 32 * NW * MPB;
    const int items = ceildiv(bound, MPB);
    if (max_nrhs <= 1) {
        auto k = potrs_small_kernel<T, NC, NW, 1>;
        k<<<grid_for(k, threads, items, persistent), threads, 0, s>>>(wl, sz, upper, A, B);
    } else if (max_nrhs <= 4) {
        auto k = potrs_small_kernel<T, NC, NW, 4>;
        k<<<grid_for(k, threads, items, persistent), threads, 0, s>>>(wl, sz, upper, A, B);
    } else {
        auto k = potrs_small_kernel<T, NC, NW, 8>;
        k<<<grid_for(k, threads, items, persistent), threads, 0, s>>>(wl, sz, upper, A, B);
    }
}

template <typename T, int NB, int NT, int CW, int CB>
static void launch_potrf_blocked(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, bool upper,
                                 T** A, int* info, cudaStream_t s) {
    auto k = potrf_blocked_kernel<T, NB, NT, CW, CB>;
    const int smem = (int)sizeof(BlockedCholShared<T, NB, NT, CW>);
    ensure_dynamic_smem((const void*)k, smem);
    k<<<grid_for(k, NT, bound, persistent, smem), NT, smem, s>>>(wl, sz, upper, A, info);
}

template <typename T, int NT>
static void launch_potrs_blocked(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, bool upper,
                                 T** A, T** B, int max_nrhs, cudaStream_t s) {
    if (max_nrhs <= 1) {
        auto k = potrs_blocked_kernel<T, NT, 1>;
        k<<<grid_for(k, NT, bound, persistent), NT, 0, s>>>(wl, sz, upper, A, B);
    } else if (max_nrhs <= 4) {
        auto k = potrs_blocked_kernel<T, NT, 4>;
        k<<<grid_for(k, NT, bound, persistent), NT, 0, s>>>(wl, sz, upper, A, B);
    } else {
        auto k = potrs_blocked_kernel<T, NT, 8>;
        k<<<grid_for(k, NT, bound, persistent), NT, 0, s>>>(wl, sz, upper, A, B);
    }
}

// Size buckets shared by the Cholesky launchers (upper edges, inclusive).
const int kCholEdges[kCholBuckets] = {8, 16, 32, 64, 128, 256, 512, 1024};

template <typename T>
void chol_bucket(int b, const WorkList& wl, int bound, bool persistent, const LuSizes& sz, bool upper, T** A, T** B,
                 int* info, bool factor, bool solve, int max_nrhs, cudaStream_t s) {
    if (factor) {
        switch (b) {
            case 0: launch_chol_small<T, 8, 1>(wl, bound, persistent, sz, upper, A, B, info, solve, max_nrhs, s); break;
            case 1: launch_chol_small<T, 16, 1>(wl, bound, persistent, sz, upper, A, B, info, solve, max_nrhs, s); break;
            case 2: launch_chol_small<T, 32, 1>(wl, bound, persistent, sz, upper, A, B, info, solve, max_nrhs, s); break;
            case 3: launch_chol_small<T, 64, 2>(wl, bound, persistent, sz, upper, A, B, info, solve, max_nrhs, s); break;
            case 4: launch_potrf_blocked<T, 32, 128, 64, 8>(wl, bound, persistent, sz, upper, A, info, s); break;
            case 5: launch_potrf_blocked<T, 32, 256, 64, 8>(wl, bound, persistent, sz, upper, A, info, s); break;
            case 6: launch_potrf_blocked<T, 32, 512, 64, 8>(wl, bound, persistent, sz, upper, A, info, s); break;
            default: launch_potrf_blocked<T, 16, 1024, 64, 4>(wl, bound, persistent, sz, upper, A, info, s); break;
        }
        if (!solve || b <= 3) return;   // small buckets fuse the solve into the factor kernel
    }
    switch (b) {
        case 0: launch_potrs_small<T, 8, 1>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
        case 1: launch_potrs_small<T, 16, 1>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
        case 2: launch_potrs_small<T, 32, 1>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
        case 3: launch_potrs_small<T, 64, 2>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
        case 4: launch_potrs_blocked<T, 128>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
        case 5: launch_potrs_blocked<T, 256>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
        case 6: launch_potrs_blocked<T, 512>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
        default: launch_potrs_blocked<T, 1024>(wl, bound, persistent, sz, upper, A, B, max_nrhs, s); break;
    }
}

int chol_bucket_of(int n) {
    for (int b = 0; b < kCholBuckets; ++b)
        if (n <= kCholEdges[b]) return b;
    return -1;
}

template void chol_bucket<double>(int, const WorkList&, int, bool, const LuSizes&, bool, double**, double**, int*, bool,
                                  bool, int, cudaStream_t);
template void chol_bucket<float>(int, const WorkList&, int, bool, const LuSizes&, bool, float**, float**, int*, bool,
                                 bool, int, cudaStream_t);

}  // namespace mb200
