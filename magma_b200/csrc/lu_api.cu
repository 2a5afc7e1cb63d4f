// lu_api.cu -- C-ABI entry points of the batched LU path.
//
// Argument checking, error codes and the info_array contract follow the
// reference drivers cited per function. The call path performs no cudaMalloc,
// no host synchronisation and no device-to-host copy.
#include "batched_kernels.h"
#include <algorithm>

using namespace mb200;

namespace {

template <typename T>
magma_int_t getrf_impl(const char* name, magma_int_t m, magma_int_t n, T** dA_array, magma_int_t ldda,
                       magma_int_t** ipiv_array, magma_int_t* info_array, magma_int_t batchCount,
                       magma_queue_t queue) {
    if (batchCount > 0) cudaMemsetAsync(info_array, 0, sizeof(magma_int_t) * batchCount, queue->stream);
    magma_int_t arginfo = 0;
    if (m < 0) arginfo = -1;
    else if (n < 0) arginfo = -2;
    else if (ldda < std::max(1, m)) arginfo = -4;
    if (arginfo != 0) {
        magma_xerbla(name, -arginfo);
        return arginfo;
    }
    if (m == 0 || n == 0 || batchCount <= 0) return 0;
    const WorkList wl{nullptr, nullptr, batchCount};
    const LuSizes sz{m, n, ldda, 0, 0, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (small_lu_supported(m, n))
        return getrf_small<T>(wl, batchCount, false, sz, m, n, dA_array, ipiv_array, info_array, queue->stream);
    if (blocked_lu_supported(m))
        return getrf_blocked<T>(wl, batchCount, false, sz, m, dA_array, ipiv_array, info_array, queue->stream);
    return MAGMA_ERR_NOT_SUPPORTED;
}

template <typename T>
magma_int_t getrs_impl(const char* name, magma_trans_t trans, magma_int_t n, magma_int_t nrhs, T** dA_array,
                       magma_int_t ldda, magma_int_t** dipiv_array, T** dB_array, magma_int_t lddb,
                       magma_int_t batchCount, magma_queue_t queue) {
    const bool notran = (trans == MagmaNoTrans);
    magma_int_t info = 0;
    if (!notran && trans != MagmaTrans && trans != MagmaConjTrans) info = -1;
    else if (n < 0) info = -2;
    else if (nrhs < 0) info = -3;
    else if (ldda < std::max(1, n)) info = -5;
    else if (lddb < std::max(1, n)) info = -8;
    if (info != 0) {
        magma_xerbla(name, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    const WorkList wl{nullptr, nullptr, batchCount};
    const LuSizes sz{n, n, ldda, lddb, nrhs, nullptr, nullptr, nullptr, nullptr, nullptr};
    if (small_lu_supported(n, n))
        return getrs_small<T>(wl, batchCount, false, !notran, sz, n, nrhs, dA_array, dipiv_array, dB_array,
                              queue->stream);
    if (blocked_lu_supported(n))
        return getrs_blocked<T>(wl, batchCount, false, !notran, sz, n, nrhs, dA_array, dipiv_array, dB_array,
                                queue->stream);
    return MAGMA_ERR_NOT_SUPPORTED;
}

template <typename T>
magma_int_t gesv_impl(const char* name, const char* getrf_name, const char* getrs_name, magma_int_t n,
                      magma_int_t nrhs, T** dA_array, magma_int_t ldda, magma_int_t** dipiv_array, T** dB_array,
                      magma_int_t lddb, magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t info = 0;
    if (n < 0) info = -1;
    else if (nrhs < 0) info = -2;
    else if (ldda < std::max(1, n)) info = -4;
    else if (lddb < std::max(1, n)) info = -6;
    if (info != 0) {
        magma_xerbla(name, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    if (small_lu_supported(n, n)) {
        const WorkList wl{nullptr, nullptr, batchCount};
        const LuSizes sz{n, n, ldda, lddb, nrhs, nullptr, nullptr, nullptr, nullptr, nullptr};
        return gesv_small<T>(wl, batchCount, false, sz, n, nrhs, dA_array, dipiv_array, dB_array, dinfo_array,
                             queue->stream);
    }
    queue_stage_begin(queue);   // stages: getrf, getrs
    info = getrf_impl<T>(getrf_name, n, n, dA_array, ldda, dipiv_array, dinfo_array, batchCount, queue);
    if (info != MAGMA_SUCCESS) return info;
    queue_stage_mark(queue);
    info = getrs_impl<T>(getrs_name, MagmaNoTrans, n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb,
                         batchCount, queue);
    queue_stage_mark(queue);
    return info;
}

}  // namespace

extern "C" {

// src/zgetrf_batched.cpp:83-107: info_array is zeroed first, then m < 0 -> -1,
// n < 0 -> -2, ldda < max(1,m) -> -4; quick return when min(m,n) == 0.
magma_int_t magma_dgetrf_batched(magma_int_t m, magma_int_t n, double** dA_array, magma_int_t ldda,
                                 magma_int_t** ipiv_array, magma_int_t* info_array,
                                 magma_int_t batchCount, magma_queue_t queue) {
    return getrf_impl<double>(__func__, m, n, dA_array, ldda, ipiv_array, info_array, batchCount, queue);
}

// src/zgetrs_batched.cpp:87-118: trans -> -1, n -> -2, nrhs -> -3,
// ldda < max(1,n) -> -5, lddb < max(1,n) -> -8; quick return for n or nrhs 0.
magma_int_t magma_dgetrs_batched(magma_trans_t trans, magma_int_t n, magma_int_t nrhs,
                                 double** dA_array, magma_int_t ldda, magma_int_t** dipiv_array,
                                 double** dB_array, magma_int_t lddb,
                                 magma_int_t batchCount, magma_queue_t queue) {
    return getrs_impl<double>(__func__, trans, n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb, batchCount,
                              queue);
}

// src/zgesv_batched.cpp:93-147: n -> -1, nrhs -> -2, ldda -> -4, lddb -> -6.
// Like the reference, the solve runs for every instance whatever its info.
magma_int_t magma_dgesv_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                magma_int_t** dipiv_array, double** dB_array, magma_int_t lddb,
                                magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue) {
    return gesv_impl<double>(__func__, "magma_dgetrf_batched", "magma_dgetrs_batched", n, nrhs, dA_array, ldda,
                             dipiv_array, dB_array, lddb, dinfo_array, batchCount, queue);
}

// LU without pivoting (src/zgetrf_nopiv_batched.cpp:76-94: m -1, n -2, ldda -4).
// The same kernels as magma_dgetrf_batched with the pivot search replaced by the
// diagonal; info_array = first zero pivot (1-based), which is then not divided by.
magma_int_t magma_dgetrf_nopiv_batched(magma_int_t m, magma_int_t n, double** dA_array, magma_int_t ldda,
                                       magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue) {
    return getrf_impl<double>(__func__, m, n, dA_array, ldda, nullptr, info_array, batchCount, queue);
}

// src/zgetrs_nopiv_batched.cpp:89-113: trans -1, n -2, nrhs -3, ldda -5, lddb -8.
// info_array is accepted for the reference's signature and set to 0.
magma_int_t magma_dgetrs_nopiv_batched(magma_trans_t trans, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                       magma_int_t ldda, double** dB_array, magma_int_t lddb,
                                       magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue) {
    if (info_array && batchCount > 0) cudaMemsetAsync(info_array, 0, sizeof(magma_int_t) * batchCount, queue->stream);
    return getrs_impl<double>(__func__, trans, n, nrhs, dA_array, ldda, nullptr, dB_array, lddb, batchCount, queue);
}

// src/zgesv_nopiv_batched.cpp:87-104: n -1, nrhs -2, ldda -4, lddb -6.
magma_int_t magma_dgesv_nopiv_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                      double** dB_array, magma_int_t lddb, magma_int_t* info_array,
                                      magma_int_t batchCount, magma_queue_t queue) {
    return gesv_impl<double>(__func__, "magma_dgetrf_nopiv_batched", "magma_dgetrs_nopiv_batched", n, nrhs, dA_array,
                             ldda, nullptr, dB_array, lddb, info_array, batchCount, queue);
}

// Single precision: the s-variants MAGMA generates from the same z-templates
// (src/zgetrf_batched.cpp:83, src/zgetrs_batched.cpp:87, src/zgesv_batched.cpp:93).
magma_int_t magma_sgetrf_batched(magma_int_t m, magma_int_t n, float** dA_array, magma_int_t ldda,
                                 magma_int_t** ipiv_array, magma_int_t* info_array, magma_int_t batchCount,
                                 magma_queue_t queue) {
    return getrf_impl<float>(__func__, m, n, dA_array, ldda, ipiv_array, info_array, batchCount, queue);
}
magma_int_t magma_sgetrs_batched(magma_trans_t trans, magma_int_t n, magma_int_t nrhs, float** dA_array,
                                 magma_int_t ldda, magma_int_t** dipiv_array, float** dB_array, magma_int_t lddb,
                                 magma_int_t batchCount, magma_queue_t queue) {
    return getrs_impl<float>(__func__, trans, n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb, batchCount,
                             queue);
}
magma_int_t magma_sgesv_batched(magma_int_t n, magma_int_t nrhs, float** dA_array, magma_int_t ldda,
                                magma_int_t** dipiv_array, float** dB_array, magma_int_t lddb,
                                magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue) {
    return gesv_impl<float>(__func__, "magma_sgetrf_batched", "magma_sgetrs_batched", n, nrhs, dA_array, ldda,
                            dipiv_array, dB_array, lddb, dinfo_array, batchCount, queue);
}

// No batched counterpart in MAGMA 2.2 (mixed precision exists only for one
// matrix, magma_dsgesv_gpu, src/zcgesv_gpu.cpp:144). Arguments follow
// magma_dgesv_batched plus the solution and iteration arrays; checks:
// n -1, nrhs -2, ldda -4, lddb -7, lddx -9. iter_array[i] as magma_dsgesv_gpu:
// >= 0 refinement iterations used, -2 overflow converting to single, -3
// singular in single precision, -31 refinement did not converge; for negative
// iter the solve was redone in double precision (A then holds the double
// factors, info the double getrf info).
magma_int_t magma_dsgesv_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                 magma_int_t** dipiv_array, double** dB_array, magma_int_t lddb, double** dX_array,
                                 magma_int_t lddx, magma_int_t* iter_array, magma_int_t* dinfo_array,
                                 magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t info = 0;
    if (n < 0) info = -1;
    else if (nrhs < 0) info = -2;
    else if (ldda < std::max(1, n)) info = -4;
    else if (lddb < std::max(1, n)) info = -7;
    else if (lddx < std::max(1, n)) info = -9;
    if (info != 0) {
        magma_xerbla(__func__, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    return dsgesv_batched(n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb, dX_array, lddx, iter_array,
                          dinfo_array, batchCount, queue);
}

}  // extern "C"
