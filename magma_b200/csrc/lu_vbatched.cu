// lu_vbatched.cu -- variable-size batched LU: getrf / getrs / gesv with per-instance
// sizes. No counterpart in MAGMA 2.2 (its only vbatched LAPACK routine is potrf,
// include/magma_zvbatched.h:29-70); defined by analogy with magma_zpotrf_vbatched:
// size arrays of batchCount+1 device entries, a checked form that reduces the sizes
// on the device (one host synchronisation) and a _max_nocheck form that never
// synchronises. Instances are counting-sorted on the device into size buckets by
// max(m, n) and each bucket runs the kernel family for its size (register-resident
// up to 64, blocked up to 1024), walking its device list.
#include "internal.h"
#include "batched_kernels.h"
#include "vbatched.h"
#include "tuning.h"
#include <algorithm>
#include <type_traits>

namespace mb200 {

constexpr int kLuBuckets = 8;
static const int kLuEdges[kLuBuckets] = {8, 16, 32, 64, 128, 256, 512, 1024};

static int lu_bucket_of(int v) {
    for (int b = 0; b < kLuBuckets; ++b)
        if (v <= kLuEdges[b]) return b;
    return -1;
}

enum class LuOp { Getrf, Getrs, Gesv };

template <typename T>
static magma_int_t lu_var(LuOp op, bool trans, const int* m, const int* n, const int* nrhs, T** A, const int* lda,
                          int** ipiv, T** B, const int* ldb, int* info, int batch, int max_mn, int max_nrhs,
                          magma_queue_t queue) {
    const int top = lu_bucket_of(max_mn);
    if (top < 0) return MAGMA_ERR_NOT_SUPPORTED;
    const size_t bw = bucketize_ws_ints(batch, kLuBuckets);
    int* ws = static_cast<int*>(queue_workspace(queue, sizeof(int) * (bw + bucket_sort_ws_ints(batch, kLuBuckets))));
    if (!ws) return MAGMA_ERR_DEVICE_ALLOC;
    if (info) cudaMemsetAsync(info, 0, sizeof(int) * batch, queue->stream);   // empty instances
    int *counts, *lists;
    magma_int_t rc = bucketize2(m, op == LuOp::Getrf ? n : nullptr, batch, kLuEdges, kLuBuckets, queue->stream, ws,
                                &counts, &lists);
    if (!rc)
        rc = sort_buckets_desc(m, op == LuOp::Getrf ? n : nullptr, batch, kLuEdges, kLuBuckets, queue->stream, counts,
                               lists, ws + bw);
    if (rc) return rc;
    const LuSizes sz{0, 0, 0, 0, 0, m, n, lda, ldb, nrhs};
    if constexpr (std::is_same<T, double>::value) {
        if (op != LuOp::Getrs && tuning().lu_queue) {
            // orders <= 512: one persistent launch over all buckets, largest first; the
            // 1024-thread bucket (512 < max(m, n) <= 1024) beside it on an auxiliary stream
            const bool solve = op == LuOp::Gesv;
            int* head = counts + kLuBuckets;
            if (top < kLuBuckets - 1) {
                lu_queue<T>(solve, counts, lists, batch, top, head, sz, A, ipiv, B, info, max_nrhs, queue->stream);
                return launch_status();
            }
            if ((rc = queue_fork(queue))) return rc;
            const int b = kLuBuckets - 1;
            const WorkList wl{lists + (size_t)b * batch, counts + b, 0};
            cudaStream_t s0 = queue_aux(queue, 0);
            rc = getrf_blocked<T>(wl, batch, true, sz, kLuEdges[b], A, ipiv, info, s0);
            if (!rc && solve) rc = getrs_blocked<T>(wl, batch, true, false, sz, kLuEdges[b], max_nrhs, A, ipiv, B, s0);
            lu_queue<T>(solve, counts, lists, batch, top, head, sz, A, ipiv, B, info, max_nrhs, queue_aux(queue, 1));
            queue_join(queue);
            return rc ? rc : launch_status();
        }
    }
    // buckets are independent: each runs on its own auxiliary stream
    if ((rc = queue_fork(queue))) return rc;
    for (int b = top; b >= 0; --b) {
        cudaStream_t s = queue_aux(queue, top - b);
        const WorkList wl{lists + (size_t)b * batch, counts + b, 0};
        const int e = kLuEdges[b];
        if (e <= 64) {
            if (op == LuOp::Getrf) rc = getrf_small<T>(wl, batch, true, sz, e, e, A, ipiv, info, s);
            else if (op == LuOp::Gesv) rc = gesv_small<T>(wl, batch, true, sz, e, max_nrhs, A, ipiv, B, info, s);
            else rc = getrs_small<T>(wl, batch, true, trans, sz, e, max_nrhs, A, ipiv, B, s);
        } else {
            if (op != LuOp::Getrs) rc = getrf_blocked<T>(wl, batch, true, sz, e, A, ipiv, info, s);
            if (!rc && op != LuOp::Getrf)
                rc = getrs_blocked<T>(wl, batch, true, trans, sz, e, max_nrhs, A, ipiv, B, s);
        }
        if (rc) break;
    }
    queue_join(queue);
    return rc ? rc : launch_status();
}

// Device-side checks of two size arrays: some a < 0 -> code_a, some b < 0 -> code_b.
static magma_int_t check_sizes(const int* a, const int* b, int batch, magma_queue_t queue, int code_a, int code_b,
                               int out[6]) {
    magma_int_t rc = reduce_sizes(a, b, nullptr, batch, queue, out);
    if (rc) return rc;
    if (out[3] < 0) return code_a;
    if (b && out[4] < 0) return code_b;
    return 0;
}

}  // namespace mb200

using namespace mb200;

extern "C" {

magma_int_t magma_dgetrf_vbatched_max_nocheck(magma_int_t* m, magma_int_t* n, double** dA_array, magma_int_t* ldda,
                                              magma_int_t** ipiv_array, magma_int_t* info_array,
                                              magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                              magma_queue_t queue) {
    if (batchCount <= 0) return 0;
    if (max_m <= 0 || max_n <= 0) {
        cudaMemsetAsync(info_array, 0, sizeof(int) * batchCount, queue->stream);
        return 0;
    }
    return lu_var<double>(LuOp::Getrf, false, m, n, nullptr, dA_array, ldda, ipiv_array, nullptr, nullptr, info_array,
                          batchCount, std::max(max_m, max_n), 1, queue);
}

// Checks: m -1, n -2, ldda < m -4, batchCount -7 (magma_zgetrf_batched's numbering).
magma_int_t magma_dgetrf_vbatched(magma_int_t* m, magma_int_t* n, double** dA_array, magma_int_t* ldda,
                                  magma_int_t** ipiv_array, magma_int_t* info_array, magma_int_t batchCount,
                                  magma_queue_t queue) {
    magma_int_t arginfo = 0;
    int r[6] = {0, 0, 0, 0, 0, 0};
    if (batchCount < 0) arginfo = -7;
    else if (batchCount > 0) {
        magma_int_t rc = check_sizes(m, n, batchCount, queue, -1, -2, r);
        if (rc < -100) return rc;
        arginfo = rc;
        int slack = 0;
        if (!arginfo && (rc = ld_slack(m, ldda, batchCount, queue, &slack)) != 0) return rc;
        if (!arginfo && slack < 0) arginfo = -4;
    }
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    return magma_dgetrf_vbatched_max_nocheck(m, n, dA_array, ldda, ipiv_array, info_array, batchCount, r[0], r[1],
                                             queue);
}

magma_int_t magma_dgetrs_vbatched_max_nocheck(magma_trans_t trans, magma_int_t* n, magma_int_t* nrhs,
                                              double** dA_array, magma_int_t* ldda, magma_int_t** dipiv_array,
                                              double** dB_array, magma_int_t* lddb, magma_int_t batchCount,
                                              magma_int_t max_n, magma_int_t max_nrhs, magma_queue_t queue) {
    if (batchCount <= 0 || max_n <= 0 || max_nrhs <= 0) return 0;
    return lu_var<double>(LuOp::Getrs, trans != MagmaNoTrans, n, n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb,
                          nullptr, batchCount, max_n, max_nrhs, queue);
}

// Checks: trans -1, n -2, nrhs -3, ldda < n -5, lddb < n -8, batchCount -10.
magma_int_t magma_dgetrs_vbatched(magma_trans_t trans, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                  magma_int_t* ldda, magma_int_t** dipiv_array, double** dB_array, magma_int_t* lddb,
                                  magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t arginfo = 0;
    int r[6] = {0, 0, 0, 0, 0, 0};
    if (trans != MagmaNoTrans && trans != MagmaTrans && trans != MagmaConjTrans) arginfo = -1;
    else if (batchCount < 0) arginfo = -10;
    else if (batchCount > 0) {
        magma_int_t rc = check_sizes(n, nrhs, batchCount, queue, -2, -3, r);
        if (rc < -100) return rc;
        arginfo = rc;
        int sa = 0, sb = 0;
        if (!arginfo && (rc = ld_slack(n, ldda, batchCount, queue, &sa)) != 0) return rc;
        if (!arginfo && sa < 0) arginfo = -5;
        if (!arginfo && (rc = ld_slack(n, lddb, batchCount, queue, &sb)) != 0) return rc;
        if (!arginfo && sb < 0) arginfo = -8;
    }
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    return magma_dgetrs_vbatched_max_nocheck(trans, n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb, batchCount,
                                             r[0], r[1], queue);
}

magma_int_t magma_dgesv_vbatched_max_nocheck(magma_int_t* n, magma_int_t* nrhs, double** dA_array, magma_int_t* ldda,
                                             magma_int_t** dipiv_array, double** dB_array, magma_int_t* lddb,
                                             magma_int_t* dinfo_array, magma_int_t batchCount, magma_int_t max_n,
                                             magma_int_t max_nrhs, magma_queue_t queue) {
    if (batchCount <= 0) return 0;
    if (max_n <= 0 || max_nrhs <= 0) {
        cudaMemsetAsync(dinfo_array, 0, sizeof(int) * batchCount, queue->stream);
        return 0;
    }
    return lu_var<double>(LuOp::Gesv, false, n, n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb, dinfo_array,
                          batchCount, max_n, max_nrhs, queue);
}

// Checks: n -1, nrhs -2, ldda < n -4, lddb < n -7, batchCount -9.
magma_int_t magma_dgesv_vbatched(magma_int_t* n, magma_int_t* nrhs, double** dA_array, magma_int_t* ldda,
                                 magma_int_t** dipiv_array, double** dB_array, magma_int_t* lddb,
                                 magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t arginfo = 0;
    int r[6] = {0, 0, 0, 0, 0, 0};
    if (batchCount < 0) arginfo = -9;
    else if (batchCount > 0) {
        magma_int_t rc = check_sizes(n, nrhs, batchCount, queue, -1, -2, r);
        if (rc < -100) return rc;
        arginfo = rc;
        int sa = 0, sb = 0;
        if (!arginfo && (rc = ld_slack(n, ldda, batchCount, queue, &sa)) != 0) return rc;
        if (!arginfo && sa < 0) arginfo = -4;
        if (!arginfo && (rc = ld_slack(n, lddb, batchCount, queue, &sb)) != 0) return rc;
        if (!arginfo && sb < 0) arginfo = -7;
    }
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    return magma_dgesv_vbatched_max_nocheck(n, nrhs, dA_array, ldda, dipiv_array, dB_array, lddb, dinfo_array,
                                            batchCount, r[0], r[1], queue);
}

}  // extern "C"
