// lu_api.cu -- C-ABI entry points of the batched LU path.
//
// Argument checking, error codes and the info_array contract follow the
// reference drivers cited per function. The call path performs no cudaMalloc,
// no host synchronisation and no device-to-host copy.
#include "batched_kernels.h"
#include <algorithm>

using namespace mb200;

extern "C" {

// src/zgetrf_batched.cpp:83-107: info_array is zeroed first, then m < 0 -> -1,
// n < 0 -> -2, ldda < max(1,m) -> -4; quick return when min(m,n) == 0.
magma_int_t magma_dgetrf_batched(magma_int_t m, magma_int_t n, double** dA_array, magma_int_t ldda,
                                 magma_int_t** ipiv_array, magma_int_t* info_array,
                                 magma_int_t batchCount, magma_queue_t queue) {
    if (batchCount > 0) cudaMemsetAsync(info_array, 0, sizeof(magma_int_t) * batchCount, queue->stream);
    magma_int_t arginfo = 0;
    if (m < 0) arginfo = -1;
    else if (n < 0) arginfo = -2;
    else if (ldda < std::max(1, m)) arginfo = -4;
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    if (m == 0 || n == 0 || batchCount <= 0) return 0;
    if (small_lu_supported(m, n))
        return getrf_small<double>(m, n, nullptr, nullptr, ldda, nullptr, m, n, dA_array,
                                   ipiv_array, info_array, batchCount, queue->stream);
    if (blocked_lu_supported(m))
        return getrf_blocked<double>(m, n, nullptr, nullptr, ldda, nullptr, m, n, dA_array,
                                     ipiv_array, info_array, batchCount, queue->stream);
    return MAGMA_ERR_NOT_SUPPORTED;
}

// src/zgetrs_batched.cpp:87-118: trans -> -1, n -> -2, nrhs -> -3,
// ldda < max(1,n) -> -5, lddb < max(1,n) -> -8; quick return for n or nrhs 0.
magma_int_t magma_dgetrs_batched(magma_trans_t trans, magma_int_t n, magma_int_t nrhs,
                                 double** dA_array, magma_int_t ldda, magma_int_t** dipiv_array,
                                 double** dB_array, magma_int_t lddb,
                                 magma_int_t batchCount, magma_queue_t queue) {
    const bool notran = (trans == MagmaNoTrans);
    magma_int_t info = 0;
    if (!notran && trans != MagmaTrans && trans != MagmaConjTrans) info = -1;
    else if (n < 0) info = -2;
    else if (nrhs < 0) info = -3;
    else if (ldda < std::max(1, n)) info = -5;
    else if (lddb < std::max(1, n)) info = -8;
    if (info != 0) {
        magma_xerbla(__func__, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    if (small_lu_supported(n, n))
        return getrs_small<double>(!notran, n, nullptr, nrhs, nullptr, ldda, nullptr, lddb, nullptr, n,
                                   nrhs, dA_array, dipiv_array, dB_array, batchCount, queue->stream);
    if (blocked_lu_supported(n))
        return getrs_blocked<double>(!notran, n, nullptr, nrhs, nullptr, ldda, nullptr, lddb, nullptr, n,
                                     nrhs, dA_array, dipiv_array, dB_array, batchCount, queue->stream);
    return MAGMA_ERR_NOT_SUPPORTED;
}

// src/zgesv_batched.cpp:93-147: n -> -1, nrhs -> -2, ldda -> -4, lddb -> -6.
// Like the reference, the solve runs for every instance whatever its info.
magma_int_t magma_dgesv_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                magma_int_t** dipiv_array, double** dB_array, magma_int_t lddb,
                                magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t info = 0;
    if (n < 0) info = -1;
    else if (nrhs < 0) info = -2;
    else if (ldda < std::max(1, n)) info = -4;
    else if (lddb < std::max(1, n)) info = -6;
    if (info != 0) {
        magma_xerbla(__func__, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    if (small_lu_supported(n, n))
        return gesv_small<double>(n, nullptr, nrhs, nullptr, ldda, nullptr, lddb, nullptr, n, nrhs,
                                  dA_array, dipiv_array, dB_array, dinfo_array, batchCount, queue->stream);
    info = magma_dgetrf_batched(n, n, dA_array, ldda, dipiv_array, dinfo_array, batchCount, queue);
    if (info != MAGMA_SUCCESS) return info;
    return magma_dgetrs_batched(MagmaNoTrans, n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb,
                                batchCount, queue);
}

}  // extern "C"
