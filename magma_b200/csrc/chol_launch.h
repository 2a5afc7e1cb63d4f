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

}  // namespace mb200
