// getrf_blocked.cu -- kernels and host dispatch of the blocked batched LU
// (one matrix per thread block, up to 1024 rows): getrf, getrs, and the
// fixed/variable-size drivers' entry into them.
#include "internal.h"
#include "blocked_lu.cuh"
#include "getrs_blocked.cuh"
#include "batched_kernels.h"
#include "lu_sizes.h"

namespace mb200 {

template <typename T, int NB, int NT, int CW, int CB>
__global__ void __launch_bounds__(NT)
getrf_blocked_kernel(LuSizes sz, T** dA_array, int** ipiv_array, int* info_array, int batch) {
    __shared__ BlockedLuShared<T, NB, NT, CW> sh;
    const int id = blockIdx.x;
    if (id >= batch) return;
    const int m = sz.get_m(id), n = sz.get_n(id), lda = sz.get_lda(id);
    if (m <= 0 || n <= 0) {
        if (threadIdx.x == 0) info_array[id] = 0;
        return;
    }
    int info;
    blocked_getrf<T, NB, NT, CW, CB>(dA_array[id], m, n, lda, ipiv_array[id], info, sh);
    if (threadIdx.x == 0) info_array[id] = info;
}

template <typename T, int NT, int R>
__global__ void __launch_bounds__(NT)
getrs_blocked_kernel(LuSizes sz, bool trans, T** dA_array, int** ipiv_array, T** dB_array, int batch) {
    __shared__ BlockedRsShared<T, NT, R> sh;
    const int id = blockIdx.x;
    if (id >= batch) return;
    const int n = sz.get_n(id), lda = sz.get_lda(id), ldb = sz.get_ldb(id), nrhs = sz.get_nrhs(id);
    if (n <= 0 || nrhs <= 0) return;
    blocked_getrs<T, NT, R>(trans, dA_array[id], n, lda, ipiv_array[id], dB_array[id], nrhs, ldb, sh);
}

bool blocked_lu_supported(int max_m) { return max_m <= 1024; }

template <typename T>
magma_int_t getrf_blocked(int m, int n, const int* m_arr, const int* n_arr, int lda, const int* lda_arr,
                          int max_m, int max_n, T** A, int** ipiv, int* info, int batch, cudaStream_t s) {
    (void)max_n;
    LuSizes sz{m, n, lda, 0, 0, m_arr, n_arr, lda_arr, nullptr, nullptr};
    if (max_m <= 128)
        getrf_blocked_kernel<T, 32, 128, 128, 16><<<batch, 128, 0, s>>>(sz, A, ipiv, info, batch);
    else if (max_m <= 256)
        getrf_blocked_kernel<T, 32, 256, 128, 8><<<batch, 256, 0, s>>>(sz, A, ipiv, info, batch);
    else if (max_m <= 512)
        getrf_blocked_kernel<T, 32, 512, 128, 8><<<batch, 512, 0, s>>>(sz, A, ipiv, info, batch);
    else
        getrf_blocked_kernel<T, 16, 1024, 128, 4><<<batch, 1024, 0, s>>>(sz, A, ipiv, info, batch);
    return launch_status();
}

template <typename T>
magma_int_t getrs_blocked(bool trans, int n, const int* n_arr, int nrhs, const int* nrhs_arr, int lda,
                          const int* lda_arr, int ldb, const int* ldb_arr, int max_n, int max_nrhs,
                          T** A, int** ipiv, T** B, int batch, cudaStream_t s) {
    LuSizes sz{n, n, lda, ldb, nrhs, n_arr, n_arr, lda_arr, ldb_arr, nrhs_arr};
#define MB200_RS(NT_)                                                                                  \
    if (max_nrhs <= 1) getrs_blocked_kernel<T, NT_, 1><<<batch, NT_, 0, s>>>(sz, trans, A, ipiv, B, batch); \
    else getrs_blocked_kernel<T, NT_, 4><<<batch, NT_, 0, s>>>(sz, trans, A, ipiv, B, batch);
    if (max_n <= 128) { MB200_RS(128) }
    else if (max_n <= 256) { MB200_RS(256) }
    else if (max_n <= 512) { MB200_RS(512) }
    else { MB200_RS(1024) }
#undef MB200_RS
    return launch_status();
}

template magma_int_t getrf_blocked<double>(int, int, const int*, const int*, int, const int*, int, int, double**, int**, int*, int, cudaStream_t);
template magma_int_t getrf_blocked<float>(int, int, const int*, const int*, int, const int*, int, int, float**, int**, int*, int, cudaStream_t);
template magma_int_t getrs_blocked<double>(bool, int, const int*, int, const int*, int, const int*, int, const int*, int, int, double**, int**, double**, int, cudaStream_t);
template magma_int_t getrs_blocked<float>(bool, int, const int*, int, const int*, int, const int*, int, const int*, int, int, float**, int**, float**, int, cudaStream_t);

}  // namespace mb200
