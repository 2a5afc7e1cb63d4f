// getrf_small.cu -- host dispatch of the register-resident batched LU family
// (kernels in small_lu_kernels.cuh, instantiated in small_lu_inst_*.cu).
#include "internal.h"
#include "small_lu_kernels.cuh"
#include "batched_kernels.h"
#include "vbatched.h"

namespace mb200 {

#define MB200_DECLARE_SMALL(T, NC, NW)                                                                            \
    extern template void launch_getrf<T, NC, NW>(const WorkList&, int, const LuSizes&, T**, int**, int*,          \
                                                 cudaStream_t);                                                   \
    extern template void launch_gesv<T, NC, NW>(const WorkList&, int, const LuSizes&, int, T**, int**, T**, int*, \
                                                cudaStream_t);                                                    \
    extern template void launch_getrs<T, NC, NW>(const WorkList&, int, const LuSizes&, bool, int, T**, int**, T**, \
                                                 cudaStream_t);
MB200_SMALL_VARIANTS(MB200_DECLARE_SMALL)

// Grid for a list of at most `bound` items handled MPB per block: one item per
// block slot for a plain batch; for a device list (length unknown on the host)
// the resident block count of the SMs, walked with a grid-stride loop.
static int small_grid(int nw, int bound, bool persistent) {
    const int mpb = (nw == 1) ? 4 : 1;
    const int items = ceildiv(bound, mpb);
    if (!persistent) return items;
    return std::max(1, std::min(items, device_sm_count() * (nw == 1 ? 3 : 4)));
}

// Dispatch on the column bound (8, 16, 32, 64) and warps per matrix (rows / 32).
#define MB200_SMALL_DISPATCH(FN, T, max_m, max_n, ...)                                        \
    do {                                                                                      \
        const int nw_ = (max_m) <= 32 ? 1 : (max_m) <= 64 ? 2 : 4;                            \
        const int nc_ = (max_n) <= 8 ? 8 : (max_n) <= 16 ? 16 : (max_n) <= 32 ? 32 : 64;      \
        const int grid_ = small_grid(nw_, bound, persistent);                                 \
        if (nw_ == 1) {                                                                       \
            if (nc_ == 8) FN<T, 8, 1>(wl, grid_, __VA_ARGS__);                                \
            else if (nc_ == 16) FN<T, 16, 1>(wl, grid_, __VA_ARGS__);                         \
            else if (nc_ == 32) FN<T, 32, 1>(wl, grid_, __VA_ARGS__);                         \
            else FN<T, 64, 1>(wl, grid_, __VA_ARGS__);                                        \
        } else if (nw_ == 2) {                                                                \
            if (nc_ <= 32) FN<T, 32, 2>(wl, grid_, __VA_ARGS__);                              \
            else FN<T, 64, 2>(wl, grid_, __VA_ARGS__);                                        \
        } else {                                                                              \
            if (nc_ <= 32) FN<T, 32, 4>(wl, grid_, __VA_ARGS__);                              \
            else FN<T, 64, 4>(wl, grid_, __VA_ARGS__);                                        \
        }                                                                                     \
    } while (0)

bool small_lu_supported(int max_m, int max_n) { return max_m <= 128 && max_n <= 64; }

template <typename T>
magma_int_t getrf_small(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, int max_m, int max_n,
                        T** A, int** ipiv, int* info, cudaStream_t s) {
    MB200_SMALL_DISPATCH(launch_getrf, T, max_m, max_n, sz, A, ipiv, info, s);
    return launch_status();
}

template <typename T>
magma_int_t gesv_small(const WorkList& wl, int bound, bool persistent, const LuSizes& sz, int max_n, int max_nrhs,
                       T** A, int** ipiv, T** B, int* info, cudaStream_t s) {
    MB200_SMALL_DISPATCH(launch_gesv, T, max_n, max_n, sz, max_nrhs, A, ipiv, B, info, s);
    return launch_status();
}

template <typename T>
magma_int_t getrs_small(const WorkList& wl, int bound, bool persistent, bool trans, const LuSizes& sz, int max_n,
                        int max_nrhs, T** A, int** ipiv, T** B, cudaStream_t s) {
    MB200_SMALL_DISPATCH(launch_getrs, T, max_n, max_n, sz, trans, max_nrhs, A, ipiv, B, s);
    return launch_status();
}

#define MB200_SMALL_HOST(T)                                                                                        \
    template magma_int_t getrf_small<T>(const WorkList&, int, bool, const LuSizes&, int, int, T**, int**, int*,     \
                                        cudaStream_t);                                                             \
    template magma_int_t gesv_small<T>(const WorkList&, int, bool, const LuSizes&, int, int, T**, int**, T**, int*, \
                                       cudaStream_t);                                                              \
    template magma_int_t getrs_small<T>(const WorkList&, int, bool, bool, const LuSizes&, int, int, T**, int**, T**, \
                                        cudaStream_t);
MB200_SMALL_HOST(double)
MB200_SMALL_HOST(float)

}  // namespace mb200
