// getrf_small.cu -- host dispatch of the register-resident batched LU family
// (kernels in small_lu_kernels.cuh, instantiated in small_lu_inst_*.cu).
#include "internal.h"
#include "small_lu_kernels.cuh"
#include "batched_kernels.h"

namespace mb200 {

#define MB200_DECLARE_SMALL(T, NC, NW)                                                              \
    extern template void launch_getrf<T, NC, NW>(const LuSizes&, T**, int**, int*, int, cudaStream_t); \
    extern template void launch_gesv<T, NC, NW>(const LuSizes&, int, T**, int**, T**, int*, int, cudaStream_t); \
    extern template void launch_getrs<T, NC, NW>(const LuSizes&, bool, int, T**, int**, T**, int, cudaStream_t);
MB200_SMALL_VARIANTS(MB200_DECLARE_SMALL)

// ---------------------------------------------------------------------------
// Host dispatch: pick (NC, NW) from the largest instance.

// Dispatch on the column bound (8, 16, 32, 64) and warps per matrix (rows / 32).
#define MB200_SMALL_DISPATCH(FN, T, max_m, max_n, ...)                            \
    do {                                                                          \
        const int nw_ = (max_m) <= 32 ? 1 : (max_m) <= 64 ? 2 : 4;               \
        const int nc_ = (max_n) <= 8 ? 8 : (max_n) <= 16 ? 16 : (max_n) <= 32 ? 32 : 64; \
        if (nw_ == 1) {                                                           \
            if (nc_ == 8) FN<T, 8, 1>(__VA_ARGS__);                               \
            else if (nc_ == 16) FN<T, 16, 1>(__VA_ARGS__);                        \
            else if (nc_ == 32) FN<T, 32, 1>(__VA_ARGS__);                        \
            else FN<T, 64, 1>(__VA_ARGS__);                                       \
        } else if (nw_ == 2) {                                                    \
            if (nc_ <= 32) FN<T, 32, 2>(__VA_ARGS__);                             \
            else FN<T, 64, 2>(__VA_ARGS__);                                       \
        } else {                                                                  \
            if (nc_ <= 32) FN<T, 32, 4>(__VA_ARGS__);                             \
            else FN<T, 64, 4>(__VA_ARGS__);                                       \
        }                                                                         \
    } while (0)

bool small_lu_supported(int max_m, int max_n) { return max_m <= 128 && max_n <= 64; }

template <typename T>
magma_int_t getrf_small(int m, int n, const int* m_arr, const int* n_arr, int lda, const int* lda_arr,
                        int max_m, int max_n, T** A, int** ipiv, int* info, int batch, cudaStream_t s) {
    LuSizes sz{m, n, lda, 0, 0, m_arr, n_arr, lda_arr, nullptr, nullptr};
    MB200_SMALL_DISPATCH(launch_getrf, T, max_m, max_n, sz, A, ipiv, info, batch, s);
    return launch_status();
}

template <typename T>
magma_int_t gesv_small(int n, const int* n_arr, int nrhs, const int* nrhs_arr, int lda, const int* lda_arr,
                       int ldb, const int* ldb_arr, int max_n, int max_nrhs, T** A, int** ipiv, T** B,
                       int* info, int batch, cudaStream_t s) {
    LuSizes sz{n, n, lda, ldb, nrhs, n_arr, n_arr, lda_arr, ldb_arr, nrhs_arr};
    MB200_SMALL_DISPATCH(launch_gesv, T, max_n, max_n, sz, max_nrhs, A, ipiv, B, info, batch, s);
    return launch_status();
}

template <typename T>
magma_int_t getrs_small(bool trans, int n, const int* n_arr, int nrhs, const int* nrhs_arr, int lda,
                        const int* lda_arr, int ldb, const int* ldb_arr, int max_n, int max_nrhs,
                        T** A, int** ipiv, T** B, int batch, cudaStream_t s) {
    LuSizes sz{n, n, lda, ldb, nrhs, n_arr, n_arr, lda_arr, ldb_arr, nrhs_arr};
    MB200_SMALL_DISPATCH(launch_getrs, T, max_n, max_n, sz, trans, max_nrhs, A, ipiv, B, batch, s);
    return launch_status();
}

template magma_int_t getrf_small<double>(int, int, const int*, const int*, int, const int*, int, int, double**, int**, int*, int, cudaStream_t);
template magma_int_t gesv_small<double>(int, const int*, int, const int*, int, const int*, int, const int*, int, int, double**, int**, double**, int*, int, cudaStream_t);
template magma_int_t getrs_small<double>(bool, int, const int*, int, const int*, int, const int*, int, const int*, int, int, double**, int**, double**, int, cudaStream_t);

}  // namespace mb200
