// lu_sizes.h -- per-instance size lookup shared by the batched kernels.
#pragma once

namespace mb200 {

// Per-instance size lookup: fixed sizes when the array pointer is null.
struct LuSizes {
    int m, n, lda, ldb, nrhs;
    const int* m_arr;
    const int* n_arr;
    const int* lda_arr;
    const int* ldb_arr;
    const int* nrhs_arr;
    __device__ __forceinline__ int get_m(int i) const { return m_arr ? m_arr[i] : m; }
    __device__ __forceinline__ int get_n(int i) const { return n_arr ? n_arr[i] : n; }
    __device__ __forceinline__ int get_lda(int i) const { return lda_arr ? lda_arr[i] : lda; }
    __device__ __forceinline__ int get_ldb(int i) const { return ldb_arr ? ldb_arr[i] : ldb; }
    __device__ __forceinline__ int get_nrhs(int i) const { return nrhs_arr ? nrhs_arr[i] : nrhs; }
};

}  // namespace mb200

namespace mb200 {

// The instances a launch works on: either 0..total-1, or the entries of a
// device list (one size bucket of a variable-size batch) whose length the
// device holds in *count. Kernels walk it with a grid-stride loop, so a
// launch never needs the length on the host.
struct WorkList {
    const int* list;
    const int* count;
    int total;
    __device__ __forceinline__ int size() const { return count ? *count : total; }
    __device__ __forceinline__ int at(int w) const { return list ? list[w] : w; }
};

}  // namespace mb200
