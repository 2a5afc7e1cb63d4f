// chol_api.cu -- C-ABI entry points of the batched Cholesky path (fixed and
// variable size). Argument checks and codes follow the reference routines
// cited per function. info_array is written for every instance (0 or the
// order of the first non-positive-definite leading minor), as LAPACK does.
#include "internal.h"
#include "chol_launch.h"
#include "vbatched.h"
#include "tuning.h"
#include <algorithm>

using namespace mb200;

namespace {

template <typename T>
magma_int_t chol_fixed(bool upper, int n, int nrhs, T** A, int lda, T** B, int ldb, int* info, int batch,
                       bool factor, bool solve, magma_queue_t queue) {
    const int b = chol_bucket_of(n);
    if (b < 0) return MAGMA_ERR_NOT_SUPPORTED;
    LuSizes sz{n, n, lda, ldb, nrhs, nullptr, nullptr, nullptr, nullptr, nullptr};
    WorkList wl{nullptr, nullptr, batch};
    chol_bucket<T>(b, wl, batch, false, sz, upper, A, B, info, factor, solve, nrhs, queue->stream);
    return launch_status();
}

// Variable size: instances are counting-sorted into size buckets on the
// device; each bucket's kernel walks its own list, the buckets concurrently.
template <typename T>
magma_int_t chol_var(bool upper, const int* n, const int* nrhs, T** A, const int* lda, T** B, const int* ldb,
                     int* info, int batch, int max_n, int max_nrhs, bool factor, bool solve, magma_queue_t queue) {
    const int top = chol_bucket_of(max_n);
    if (top < 0) return MAGMA_ERR_NOT_SUPPORTED;
    const size_t bw = bucketize_ws_ints(batch, kCholBuckets);
    int* ws = static_cast<int*>(queue_workspace(queue, sizeof(int) * (bw + bucket_sort_ws_ints(batch, kCholBuckets))));
    if (!ws) return MAGMA_ERR_DEVICE_ALLOC;
    if (info) cudaMemsetAsync(info, 0, sizeof(int) * batch, queue->stream);   // n = 0 instances
    int *counts, *lists;
    magma_int_t rc = bucketize(n, batch, kCholEdges, kCholBuckets, queue->stream, ws, &counts, &lists);
    if (!rc) rc = sort_buckets_desc(n, nullptr, batch, kCholEdges, kCholBuckets, queue->stream, counts, lists, ws + bw);
    if (rc) return rc;
    LuSizes sz{0, 0, 0, 0, 0, n, n, lda, ldb, nrhs};
    if (tuning().chol_queue) {
        // orders <= 512: one persistent launch over all buckets, largest first; the
        // 1024-thread bucket (512 < n <= 1024) beside it on an auxiliary stream
        int* head = counts + kCholBuckets;
        if (top < kCholBuckets - 1) {
            chol_queue<T>(counts, lists, batch, top, head, sz, upper, A, B, info, factor, solve, max_nrhs,
                          queue->stream);
            return launch_status();
        }
        if ((rc = queue_fork(queue))) return rc;
        const int b = kCholBuckets - 1;
        WorkList wl{lists + (size_t)b * batch, counts + b, 0};
        chol_bucket<T>(b, wl, batch, true, sz, upper, A, B, info, factor, solve, max_nrhs, queue_aux(queue, 0));
        chol_queue<T>(counts, lists, batch, top, head, sz, upper, A, B, info, factor, solve, max_nrhs,
                      queue_aux(queue, 1));
        queue_join(queue);
        return launch_status();
    }
    // buckets are independent: each runs on its own auxiliary stream
    if ((rc = queue_fork(queue))) return rc;
    for (int b = top; b >= 0; --b) {
        WorkList wl{lists + (size_t)b * batch, counts + b, 0};
        chol_bucket<T>(b, wl, batch, true, sz, upper, A, B, info, factor, solve, max_nrhs,
                       queue_aux(queue, top - b));
    }
    queue_join(queue);
    return launch_status();
}

// magmablas/vbatched_check.cu:840-892 (potrf_vbatched_checker): uplo -> -1,
// some n < 0 -> -2, some ldda < n -> -4, batchCount < 0 -> -6.
magma_int_t check_potrf_v(magma_uplo_t uplo, const int* n, const int* ldda, int batch, magma_queue_t queue,
                          int* max_n) {
    if (uplo != MagmaLower && uplo != MagmaUpper) return -1;
    if (batch < 0) return -6;
    if (batch == 0) { *max_n = 0; return 0; }
    int r[6];
    magma_int_t rc = reduce_sizes(n, nullptr, nullptr, batch, queue, r);
    if (rc) return rc;
    if (r[3] < 0) return -2;
    int slack = 0;
    rc = ld_slack(n, ldda, batch, queue, &slack);
    if (rc) return rc;
    if (slack < 0) return -4;
    *max_n = r[0];
    return 0;
}

}  // namespace

extern "C" {

// src/zpotrf_batched.cpp:291-320: info zeroed first; uplo -> -1, n -> -2, ldda -> -4.
magma_int_t magma_dpotrf_batched(magma_uplo_t uplo, magma_int_t n, double** dA_array, magma_int_t ldda,
                                 magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue) {
    if (batchCount > 0) cudaMemsetAsync(info_array, 0, sizeof(magma_int_t) * batchCount, queue->stream);
    magma_int_t arginfo = 0;
    if (uplo != MagmaUpper && uplo != MagmaLower) arginfo = -1;
    else if (n < 0) arginfo = -2;
    else if (ldda < std::max(1, n)) arginfo = -4;
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    if (n == 0 || batchCount <= 0) return 0;
    return chol_fixed<double>(uplo == MagmaUpper, n, 0, dA_array, ldda, nullptr, 0, info_array, batchCount, true,
                              false, queue);
}

// src/zpotrs_batched.cpp:71-94. The reference tests every argument and keeps
// the LAST failing one (uplo -1, n -2, nrhs -3, ldda -5, lddb -7).
magma_int_t magma_dpotrs_batched(magma_uplo_t uplo, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                 magma_int_t ldda, double** dB_array, magma_int_t lddb, magma_int_t batchCount,
                                 magma_queue_t queue) {
    magma_int_t info = 0;
    if (uplo != MagmaUpper && uplo != MagmaLower) info = -1;
    if (n < 0) info = -2;
    if (nrhs < 0) info = -3;
    if (ldda < std::max(1, n)) info = -5;
    if (lddb < std::max(1, n)) info = -7;
    if (info != 0) {
        magma_xerbla(__func__, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    return chol_fixed<double>(uplo == MagmaUpper, n, nrhs, dA_array, ldda, dB_array, lddb, nullptr, batchCount,
                              false, true, queue);
}

// src/zposv_batched.cpp:89-141 (same last-failing-argument checks as potrs).
magma_int_t magma_dposv_batched(magma_uplo_t uplo, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                magma_int_t ldda, double** dB_array, magma_int_t lddb, magma_int_t* dinfo_array,
                                magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t info = 0;
    if (uplo != MagmaUpper && uplo != MagmaLower) info = -1;
    if (n < 0) info = -2;
    if (nrhs < 0) info = -3;
    if (ldda < std::max(1, n)) info = -5;
    if (lddb < std::max(1, n)) info = -7;
    if (info != 0) {
        magma_xerbla(__func__, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    return chol_fixed<double>(uplo == MagmaUpper, n, nrhs, dA_array, ldda, dB_array, lddb, dinfo_array, batchCount,
                              true, true, queue);
}

// include/magma_zvbatched.h:59-64; src/zpotrf_vbatched.cpp:251-267.
magma_int_t magma_dpotrf_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, double** dA_array,
                                              magma_int_t* ldda, magma_int_t* info_array, magma_int_t batchCount,
                                              magma_int_t max_n, magma_queue_t queue) {
    if (batchCount <= 0 || max_n <= 0) return 0;
    return chol_var<double>(uplo == MagmaUpper, n, nullptr, dA_array, ldda, nullptr, nullptr, info_array,
                            batchCount, max_n, 0, true, false, queue);
}

// include/magma_zvbatched.h:66-70; src/zpotrf_vbatched.cpp:335-356 (checker, max_n, then _max_nocheck).
magma_int_t magma_dpotrf_vbatched(magma_uplo_t uplo, magma_int_t* n, double** dA_array, magma_int_t* ldda,
                                  magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue) {
    int max_n = 0;
    magma_int_t arginfo = check_potrf_v(uplo, n, ldda, batchCount, queue, &max_n);
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    return magma_dpotrf_vbatched_max_nocheck(uplo, n, dA_array, ldda, info_array, batchCount, max_n, queue);
}

// No counterpart in MAGMA 2.2 (potrs exists only for fixed sizes,
// src/zpotrs_batched.cpp:71); defined by analogy with magma_dpotrf_vbatched:
// per-instance n, nrhs, ldda, lddb device arrays of batchCount+1 entries.
magma_int_t magma_dpotrs_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs,
                                              double** dA_array, magma_int_t* ldda, double** dB_array,
                                              magma_int_t* lddb, magma_int_t batchCount, magma_int_t max_n,
                                              magma_int_t max_nrhs, magma_queue_t queue) {
    if (batchCount <= 0 || max_n <= 0 || max_nrhs <= 0) return 0;
    return chol_var<double>(uplo == MagmaUpper, n, nrhs, dA_array, ldda, dB_array, lddb, nullptr, batchCount,
                            max_n, max_nrhs, false, true, queue);
}

// Checks: uplo -1, n -2, nrhs -3, ldda < n -5, lddb < n -7, batchCount -9.
magma_int_t magma_dpotrs_vbatched(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                  magma_int_t* ldda, double** dB_array, magma_int_t* lddb, magma_int_t batchCount,
                                  magma_queue_t queue) {
    magma_int_t arginfo = 0;
    int r[6] = {0, 0, 0, 0, 0, 0};
    if (uplo != MagmaLower && uplo != MagmaUpper) arginfo = -1;
    else if (batchCount < 0) arginfo = -9;
    else if (batchCount > 0) {
        magma_int_t rc = reduce_sizes(n, nrhs, nullptr, batchCount, queue, r);
        if (rc) return rc;
        int sa = 0, sb = 0;
        if (r[3] < 0) arginfo = -2;
        else if (r[4] < 0) arginfo = -3;
        else if ((rc = ld_slack(n, ldda, batchCount, queue, &sa)) != 0) return rc;
        else if (sa < 0) arginfo = -5;
        else if ((rc = ld_slack(n, lddb, batchCount, queue, &sb)) != 0) return rc;
        else if (sb < 0) arginfo = -7;
    }
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    return magma_dpotrs_vbatched_max_nocheck(uplo, n, nrhs, dA_array, ldda, dB_array, lddb, batchCount, r[0], r[1],
                                             queue);
}

// No counterpart in MAGMA 2.2: potrf + potrs on variable sizes in one call
// (fused into one kernel per instance for n <= 64).
magma_int_t magma_dposv_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs,
                                             double** dA_array, magma_int_t* ldda, double** dB_array,
                                             magma_int_t* lddb, magma_int_t* dinfo_array, magma_int_t batchCount,
                                             magma_int_t max_n, magma_int_t max_nrhs, magma_queue_t queue) {
    if (batchCount <= 0) return 0;
    if (max_n <= 0) {
        cudaMemsetAsync(dinfo_array, 0, sizeof(int) * batchCount, queue->stream);
        return 0;
    }
    return chol_var<double>(uplo == MagmaUpper, n, nrhs, dA_array, ldda, dB_array, lddb, dinfo_array, batchCount,
                            max_n, std::max(max_nrhs, 1), true, true, queue);
}

magma_int_t magma_dposv_vbatched(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                 magma_int_t* ldda, double** dB_array, magma_int_t* lddb, magma_int_t* dinfo_array,
                                 magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t arginfo = 0;
    int r[6] = {0, 0, 0, 0, 0, 0};
    if (uplo != MagmaLower && uplo != MagmaUpper) arginfo = -1;
    else if (batchCount < 0) arginfo = -10;
    else if (batchCount > 0) {
        magma_int_t rc = reduce_sizes(n, nrhs, nullptr, batchCount, queue, r);
        if (rc) return rc;
        int sa = 0, sb = 0;
        if (r[3] < 0) arginfo = -2;
        else if (r[4] < 0) arginfo = -3;
        else if ((rc = ld_slack(n, ldda, batchCount, queue, &sa)) != 0) return rc;
        else if (sa < 0) arginfo = -5;
        else if ((rc = ld_slack(n, lddb, batchCount, queue, &sb)) != 0) return rc;
        else if (sb < 0) arginfo = -7;
    }
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    return magma_dposv_vbatched_max_nocheck(uplo, n, nrhs, dA_array, ldda, dB_array, lddb, dinfo_array, batchCount,
                                            r[0], r[1], queue);
}

}  // extern "C"
