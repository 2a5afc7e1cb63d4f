// batched_kernels.h -- internal launchers shared by the C-ABI entry points.
// Every launcher enqueues on `s` and returns MAGMA_SUCCESS or a MAGMA error.
#pragma once
#include "internal.h"

namespace mb200 {

// Register-resident LU family (getrf_small.cu): m <= 128, n <= 64.
bool small_lu_supported(int max_m, int max_n);

template <typename T>
magma_int_t getrf_small(int m, int n, const int* m_arr, const int* n_arr, int lda, const int* lda_arr,
                        int max_m, int max_n, T** A, int** ipiv, int* info, int batch, cudaStream_t s);
template <typename T>
magma_int_t gesv_small(int n, const int* n_arr, int nrhs, const int* nrhs_arr, int lda, const int* lda_arr,
                       int ldb, const int* ldb_arr, int max_n, int max_nrhs, T** A, int** ipiv, T** B,
                       int* info, int batch, cudaStream_t s);
template <typename T>
magma_int_t getrs_small(bool trans, int n, const int* n_arr, int nrhs, const int* nrhs_arr, int lda,
                        const int* lda_arr, int ldb, const int* ldb_arr, int max_n, int max_nrhs,
                        T** A, int** ipiv, T** B, int batch, cudaStream_t s);

// Blocked LU family (getrf_blocked.cu): one matrix per thread block, m <= 1024.
bool blocked_lu_supported(int max_m);

template <typename T>
magma_int_t getrf_blocked(int m, int n, const int* m_arr, const int* n_arr, int lda, const int* lda_arr,
                          int max_m, int max_n, T** A, int** ipiv, int* info, int batch, cudaStream_t s);
template <typename T>
magma_int_t getrs_blocked(bool trans, int n, const int* n_arr, int nrhs, const int* nrhs_arr, int lda,
                          const int* lda_arr, int ldb, const int* ldb_arr, int max_n, int max_nrhs,
                          T** A, int** ipiv, T** B, int batch, cudaStream_t s);

}  // namespace mb200
