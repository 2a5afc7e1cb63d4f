// batched_kernels.h -- internal launchers shared by the C-ABI entry points.
// Every launcher enqueues on `s` and returns MAGMA_SUCCESS or a MAGMA error.
// `wl` lists the instances to process and `bound` bounds its length; with
// `persistent` the grid is capped at the resident block count and the kernel
// walks the list (used when the list lives on the device).
#pragma once
#include "internal.h"
#include "lu_sizes.h"

namespace mb200 {

// Register-resident LU family (getrf_small.cu): m <= 128, n <= 64.
bool small_lu_supported(int max_m, int max_n);
template <typename T>
magma_int_t getrf_small(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, int max_m, int max_n,
                        T** A, int** ipiv, int* info, cudaStream_t s);
template <typename T>
magma_int_t gesv_small(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, int max_n, int max_nrhs,
                       T** A, int** ipiv, T** B, int* info, cudaStream_t s);
template <typename T>
magma_int_t getrs_small(const WorkList& wl, int bound, bool persistent, bool trans, const LuSizes& sz, int max_n,
                        int max_nrhs, T** A, int** ipiv, T** B, cudaStream_t s);

// Blocked LU family (getrf_blocked.cu): one matrix per thread block, m <= 1024.
bool blocked_lu_supported(int max_m);
template <typename T>
magma_int_t getrf_blocked(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, int max_m, T** A,
                          int** ipiv, int* info, cudaStream_t s);
template <typename T>
magma_int_t getrs_blocked(const WorkList& wl, int bound, bool persistent, bool trans, const LuSizes& sz, int max_n,
                          int max_nrhs, T** A, int** ipiv, T** B, cudaStream_t s);

// One launch for buckets min(top, 6)..0 of a bucketize() result keyed by max(m, n)
// (orders up to 512): the persistent queue kernel of lu_queue.cuh. getrf when !solve,
// else gesv (getrf + getrs NoTrans). `head` must hold 0 (ticket counter). Same work
// and results as the per-bucket getrf / gesv kernels over those buckets.
template <typename T>
void lu_queue(bool solve, const int* counts, const int* lists, int batch, int top, int* head, const LuSizes& sz,
              T** A, int** ipiv, T** B, int* info, int max_nrhs, cudaStream_t s);

// Mixed-precision LU solve (mixed.cu): FP32 factor, FP64 refinement, FP64 fallback; n <= 512.
bool dsgesv_supported(int n);
magma_int_t dsgesv_batched(int n, int nrhs, double** dA, int lda, int** ipiv, double** dB, int ldb, double** dX,
                           int ldx, int* iter, int* info, int batch, magma_queue_t queue);

}  // namespace mb200
