// lu_queue.cu -- host launcher of the one-launch variable-size LU (device code and
// design in lu_queue.cuh).
#include "internal.h"
#include "lu_queue.cuh"
#include "batched_kernels.h"
#include "vbatched.h"

namespace mb200 {

template <typename T, bool SOLVE, int R>
static void launch_lu_queue(const LuQueue& q, int bound, const LuSizes& sz, T** A, int** ipiv, T** B, int* info,
                            cudaStream_t s) {
    auto k = lu_queue_kernel<T, SOLVE, R>;
    const size_t smem = LuQueueShare<T, R>::bytes * kLuQueueWarps;
    ensure_dynamic_smem((const void*)k, (int)smem);
    const int grid = max(1, min(bound, resident_blocks((const void*)k, kLuQueueThreads, smem)));
    k<<<grid, kLuQueueThreads, smem, s>>>(q, sz, A, ipiv, B, info);
}

template <typename T>
void lu_queue(bool solve, const int* counts, const int* lists, int batch, int top, int* head, const LuSizes& sz,
              T** A, int** ipiv, T** B, int* info, int max_nrhs, cudaStream_t s) {
    const LuQueue q{counts, lists, batch, min(top, kLuQueueBuckets - 1), head};
    if (!solve) launch_lu_queue<T, false, 1>(q, batch, sz, A, ipiv, B, info, s);
    else if (max_nrhs <= 1) launch_lu_queue<T, true, 1>(q, batch, sz, A, ipiv, B, info, s);
    else launch_lu_queue<T, true, 4>(q, batch, sz, A, ipiv, B, info, s);
}

template void lu_queue<double>(bool, const int*, const int*, int, int, int*, const LuSizes&, double**, int**,
                               double**, int*, int, cudaStream_t);

}  // namespace mb200
