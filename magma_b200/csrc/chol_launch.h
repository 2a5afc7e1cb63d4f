// chol_launch.h -- host launchers of the batched Cholesky kernels.
#pragma once
#include "internal.h"
#include "lu_sizes.h"

namespace mb200 {

constexpr int kCholBuckets = 8;
extern const int kCholEdges[kCholBuckets];   // {8, 16, 32, 64, 128, 256, 512, 1024}

// Bucket index of an order n (-1 when n > 1024).
int chol_bucket_of(int n);

// Launches bucket b's kernels over the instances of `wl`: potrf when `factor`,
// potrs when `solve` (fused into one kernel for n <= 64). `bound` is an upper
// bound on wl's length; `persistent` caps the grid at the resident block
// count (the kernels walk the list with a grid-stride loop).
template <typename T>
void chol_bucket(int b, const WorkList& wl, int bound, bool persistent, const LuSizes& sz, bool upper, T** A, T** B,
                 int* info, bool factor, bool solve, int max_nrhs, cudaStream_t s);

// One launch for buckets min(top, 6)..0 of a bucketize() result (orders up to 512):
// the persistent queue kernel of chol_queue.cuh. `head` must hold 0 and is used
// as the ticket counter. Same work and results as chol_bucket over those buckets.
template <typename T>
void chol_queue(const int* counts, const int* lists, int batch, int top, int* head, const LuSizes& sz, bool upper,
                T** A, T** B, int* info, bool factor, bool solve, int max_nrhs, cudaStream_t s);

}  // namespace mb200
