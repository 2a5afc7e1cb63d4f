// chol_queue.cu -- host launcher of the one-launch variable-size Cholesky
// (device code and design in chol_queue.cuh).
#include "internal.h"
#include "chol_queue.cuh"
#include "vbatched.h"

namespace mb200 {

template <typename T, bool FACTOR, bool SOLVE, int R>
static void launch_queue(const CholQueue& q, int bound, const LuSizes& sz, bool upper, T** A, T** B, int* info,
                         cudaStream_t s) {
    auto k = chol_queue_kernel<T, FACTOR, SOLVE, R>;
    const size_t smem = QueueShare<T, R>::bytes * kQueueWarps;
    ensure_dynamic_smem((const void*)k, (int)smem);
    const int grid = max(1, min(bound, resident_blocks((const void*)k, kQueueThreads, smem)));
    k<<<grid, kQueueThreads, smem, s>>>(q, sz, upper, A, B, info);
}

template <typename T>
void chol_queue(const int* counts, const int* lists, int batch, int top, int* head, const LuSizes& sz, bool upper,
                T** A, T** B, int* info, bool factor, bool solve, int max_nrhs, cudaStream_t s) {
    const CholQueue q{counts, lists, batch, min(top, kQueueBuckets - 1), head};
    // right-hand sides are solved in groups of R = 1, 4 or 8 (the same operations per element)
    if (factor && solve) {
        if (max_nrhs <= 1) launch_queue<T, true, true, 1>(q, batch, sz, upper, A, B, info, s);
        else if (max_nrhs <= 4) launch_queue<T, true, true, 4>(q, batch, sz, upper, A, B, info, s);
        else launch_queue<T, true, true, 8>(q, batch, sz, upper, A, B, info, s);
    } else if (factor) {
        launch_queue<T, true, false, 1>(q, batch, sz, upper, A, B, info, s);
    } else if (max_nrhs <= 1) {
        launch_queue<T, false, true, 1>(q, batch, sz, upper, A, B, info, s);
    } else if (max_nrhs <= 4) {
        launch_queue<T, false, true, 4>(q, batch, sz, upper, A, B, info, s);
    } else {
        launch_queue<T, false, true, 8>(q, batch, sz, upper, A, B, info, s);
    }
}

template void chol_queue<double>(const int*, const int*, int, int, int*, const LuSizes&, bool, double**, double**,
                                 int*, bool, bool, int, cudaStream_t);

}  // namespace mb200
