// getrf_blocked.cu -- kernels and host dispatch of the blocked batched LU
// (one matrix per thread block, up to 1024 rows): getrf and getrs.
#include "internal.h"
#include "blocked_lu.cuh"
#include "getrs_blocked.cuh"
#include "batched_kernels.h"
#include "lu_sizes.h"
#include "vbatched.h"
#include "tuning.h"

namespace mb200 {

// Resident blocks per SM the register allocation is sized for.
template <typename T, int NT>
constexpr int blocked_min_blocks() {
    return NT <= 128 ? 4 : NT == 256 ? (sizeof(T) == 8 ? 2 : 3) : 1;
}

template <typename T, int NB, int NT, int CW, int CB, bool DMMA>
__global__ void __launch_bounds__(NT, (blocked_min_blocks<T, NT>()))
getrf_blocked_kernel(WorkList wl, LuSizes sz, T** dA_array, int** ipiv_array, int* info_array) {
    extern __shared__ __align__(16) unsigned char getrf_smem[];
    BlockedLuShared<T, NB, NT, CW, DMMA>& sh = *reinterpret_cast<BlockedLuShared<T, NB, NT, CW, DMMA>*>(getrf_smem);
    for (int w = blockIdx.x; w < wl.size(); w += gridDim.x) {
        const int id = wl.at(w);
        const int m = sz.get_m(id), n = sz.get_n(id), lda = sz.get_lda(id);
        int info = 0;
        if (m > 0 && n > 0)   // a null pivot array selects LU without pivoting (getrf_nopiv)
            blocked_getrf<T, NB, NT, CW, CB, DMMA>(dA_array[id], m, n, lda, ipiv_array ? ipiv_array[id] : nullptr,
                                                  info, sh);
        if (threadIdx.x == 0) info_array[id] = info;
        __syncthreads();
    }
}

template <typename T, int NT, int R>
__global__ void __launch_bounds__(NT)
getrs_blocked_kernel(WorkList wl, LuSizes sz, bool trans, T** dA_array, int** ipiv_array, T** dB_array) {
    __shared__ BlockedRsShared<T, NT, R> sh;
    for (int w = blockIdx.x; w < wl.size(); w += gridDim.x) {
        const int id = wl.at(w);
        const int n = sz.get_n(id), lda = sz.get_lda(id), ldb = sz.get_ldb(id), nrhs = sz.get_nrhs(id);
        if (n > 0 && nrhs > 0)
            blocked_getrs<T, NT, R>(trans, dA_array[id], n, lda, ipiv_array ? ipiv_array[id] : nullptr,
                                    dB_array[id], nrhs, ldb, sh);
        __syncthreads();
    }
}

bool blocked_lu_supported(int max_m) { return max_m <= 1024; }

template <typename K>
static int blocked_grid(K kernel, int threads, int bound, bool persistent, size_t smem = 0) {
    if (!persistent) return std::max(1, bound);
    return std::max(1, std::min(bound, resident_blocks((const void*)kernel, threads, smem)));
}

template <typename T, int NB, int NT, int CW, int CB, bool DMMA>
static void launch_getrf_blocked(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, T** A, int** ipiv,
                                 int* info, cudaStream_t s) {
    auto k = getrf_blocked_kernel<T, NB, NT, CW, CB, DMMA>;
    const int smem = (int)sizeof(BlockedLuShared<T, NB, NT, CW, DMMA>);
    ensure_dynamic_smem((const void*)k, smem);
    k<<<blocked_grid(k, NT, bound, persistent, smem), NT, smem, s>>>(wl, sz, A, ipiv, info);
}

// The trailing-update variant of a bucket: FP64 on the tensor cores (DMMA) or on the
// FP64 CUDA-core pipe, as the tuning table says; FP32 always on the CUDA cores.
template <typename T, int NB, int NT, int CW, int CB>
static void launch_getrf_bucket(int bucket, const WorkList& wl, int bound, bool persistent, const LuSizes& sz, T** A,
                                int** ipiv, int* info, cudaStream_t s) {
    if (sizeof(T) == 8 && tuning().lu_dmma[bucket])
        launch_getrf_blocked<T, NB, NT, CW, CB, sizeof(T) == 8>(wl, bound, persistent, sz, A, ipiv, info, s);
    else
        launch_getrf_blocked<T, NB, NT, CW, CB, false>(wl, bound, persistent, sz, A, ipiv, info, s);
}

template <typename T>
magma_int_t getrf_blocked(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, int max_m, T** A,
                          int** ipiv, int* info, cudaStream_t s) {
    if (max_m <= 128) launch_getrf_bucket<T, 32, 128, 128, (sizeof(T) == 8 ? 8 : 16)>(0, wl, bound, persistent, sz, A, ipiv, info, s);
    else if (max_m <= 256) launch_getrf_bucket<T, 32, 256, 128, (sizeof(T) == 8 ? 4 : 8)>(1, wl, bound, persistent, sz, A, ipiv, info, s);
    else if (max_m <= 512) launch_getrf_bucket<T, 32, 512, 128, 8>(2, wl, bound, persistent, sz, A, ipiv, info, s);
    else launch_getrf_bucket<T, 16, 1024, 128, (sizeof(T) == 8 ? 2 : 4)>(3, wl, bound, persistent, sz, A, ipiv, info, s);
    return launch_status();
}

template <typename T, int NT>
static void launch_getrs_blocked(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, bool trans,
                                 int max_nrhs, T** A, int** ipiv, T** B, cudaStream_t s) {
    if (max_nrhs <= 1) {
        auto k = getrs_blocked_kernel<T, NT, 1>;
        k<<<blocked_grid(k, NT, bound, persistent), NT, 0, s>>>(wl, sz, trans, A, ipiv, B);
    } else {
        auto k = getrs_blocked_kernel<T, NT, 4>;
        k<<<blocked_grid(k, NT, bound, persistent), NT, 0, s>>>(wl, sz, trans, A, ipiv, B);
    }
}

template <typename T>
magma_int_t getrs_blocked(const WorkList& wl, int bound, bool persistent, bool trans, const LuSizes& sz, int max_n,
                          int max_nrhs, T** A, int** ipiv, T** B, cudaStream_t s) {
    if (max_n <= 128) launch_getrs_blocked<T, 128>(wl, bound, persistent, sz, trans, max_nrhs, A, ipiv, B, s);
    else if (max_n <= 256) launch_getrs_blocked<T, 256>(wl, bound, persistent, sz, trans, max_nrhs, A, ipiv, B, s);
    else if (max_n <= 512) launch_getrs_blocked<T, 512>(wl, bound, persistent, sz, trans, max_nrhs, A, ipiv, B, s);
    else launch_getrs_blocked<T, 1024>(wl, bound, persistent, sz, trans, max_nrhs, A, ipiv, B, s);
    return launch_status();
}

template magma_int_t getrf_blocked<double>(const WorkList&, int, bool, const LuSizes&, int, double**, int**, int*,
                                           cudaStream_t);
template magma_int_t getrf_blocked<float>(const WorkList&, int, bool, const LuSizes&, int, float**, int**, int*,
                                          cudaStream_t);
template magma_int_t getrs_blocked<double>(const WorkList&, int, bool, bool, const LuSizes&, int, int, double**, int**,
                                           double**, cudaStream_t);
template magma_int_t getrs_blocked<float>(const WorkList&, int, bool, bool, const LuSizes&, int, int, float**, int**,
                                          float**, cudaStream_t);

}  // namespace mb200
