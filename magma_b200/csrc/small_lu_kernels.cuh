// small_lu_kernels.cuh -- kernels of the batched LU factorisation, solve and fused gesv for
// matrices up to 128 rows x 64 columns, fixed or variable size per instance.
//
// Replaces, for these sizes, the reference's getf2 pipeline
// (src/zgetf2_batched.cpp:98-194: per column an argmax kernel, a swap kernel
// and a scale/update kernel; then laswp, trsm and gemm launches) and its
// trsv-based getrs (src/zgetrs_batched.cpp:87-273) by ONE launch each: the
// matrix is read from HBM once, factored in registers (small_lu.cuh), and
// written once.
#include "internal.h"
#include "small_lu.cuh"
#include "lu_sizes.h"

#pragma once
namespace mb200 {

// MPB matrices per block when NW == 1 (one warp each); one matrix per block otherwise.
template <int NW> struct BlockShape { static constexpr int MPB = (NW == 1) ? 4 : 1; };
// Blocks per SM the register budget is sized for (<= 128 registers a thread for NC <= 32).
template <int NC, int NW> struct MinBlocks { static constexpr int value = (NC <= 32 && NW == 1) ? 3 : 1; };

template <typename T, int NC, int NW>
__device__ __forceinline__ void load_rows(T (&a)[NC], const T* __restrict__ A, int m, int n, int lda, int tid) {
#pragma unroll
    for (int j = 0; j < NC; ++j) a[j] = (tid < m && j < n) ? A[tid + (size_t)j * lda] : T(0);
}

template <typename T, int NC>
__device__ __forceinline__ void store_rows(const T (&a)[NC], T* __restrict__ A, int m, int n, int lda, int tid, int pos) {
    if (tid < m) {
#pragma unroll
        for (int j = 0; j < NC; ++j)
            if (j < n) A[pos + (size_t)j * lda] = a[j];
    }
}

// ---------------------------------------------------------------------------
// One instance of getrf on the matrix's threads (tid = row). n <= 0 or m <= 0 writes info 0.
template <typename T, int NC, int NW>
__device__ __forceinline__ void getrf_small_instance(int id, const LuSizes& sz, T** dA_array, int** ipiv_array,
                                                     int* info_array, int tid, SmallLuShared<T, NC, NW>& sh) {
    const int m = sz.get_m(id), n = sz.get_n(id), lda = sz.get_lda(id);
    if (m <= 0 || n <= 0) {
        if (tid == 0) info_array[id] = 0;
        return;
    }
    T* A = dA_array[id];
    T a[NC];
    load_rows<T, NC, NW>(a, A, m, n, lda, tid);
    int pos, my_ipiv, info;
    // a null pivot array selects LU without pivoting (getrf_nopiv)
    small_lu_factor<T, NC, NW>(a, m, n, tid, pos, my_ipiv, info, sh, ipiv_array == nullptr);
    store_rows<T, NC>(a, A, m, n, lda, tid, pos);
    if (ipiv_array && tid < min(m, n)) ipiv_array[id][tid] = my_ipiv;
    if (tid == 0) info_array[id] = info;
}

// One instance of gesv: getrf + getrs(NoTrans) in one pass, R RHS columns solved together.
template <typename T, int NC, int NW, int R>
__device__ __forceinline__ void gesv_small_instance(int id, const LuSizes& sz, T** dA_array, int** ipiv_array,
                                                    T** dB_array, int* info_array, int tid,
                                                    SmallLuShared<T, NC, NW>& sh) {
    static_assert(R <= 4, "the shared rhs buffer holds 4 right-hand sides a group");
    const int n = sz.get_n(id), lda = sz.get_lda(id), ldb = sz.get_ldb(id), nrhs = sz.get_nrhs(id);
    if (n <= 0) {
        if (tid == 0) info_array[id] = 0;
        return;
    }
    T* A = dA_array[id];
    T* B = dB_array[id];
    T a[NC];
    load_rows<T, NC, NW>(a, A, n, n, lda, tid);
    // the first group of right-hand sides is loaded with A, so its latency hides behind
    // the factorisation (after the stores of A the compiler could not move it earlier)
    T b0[R];
#pragma unroll
    for (int r = 0; r < R; ++r) b0[r] = (tid < n && r < nrhs) ? B[tid + (size_t)r * ldb] : T(0);
    int pos, my_ipiv, info;
    small_lu_factor<T, NC, NW>(a, n, n, tid, pos, my_ipiv, info, sh, ipiv_array == nullptr);
    store_rows<T, NC>(a, A, n, n, lda, tid, pos);
    if (ipiv_array && tid < n) ipiv_array[id][tid] = my_ipiv;
    if (tid == 0) info_array[id] = info;
    // Thread tid's b entry (original row tid) belongs at position `pos` of P*b,
    // the same position its LU row landed at, so no permutation pass is needed.
    // (Every read of B happens before the first barrier of the solve, every
    // write after its last one, so rows may move between threads in place.)
    for (int c0 = 0; c0 < nrhs; c0 += R) {
        T b[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
            b[r] = (c0 == 0) ? b0[r] : (tid < n && c0 + r < nrhs) ? B[tid + (size_t)(c0 + r) * ldb] : T(0);
        small_lu_solve<T, NC, NW, R>(a, n, pos, b, sh);
        if (tid < n) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (c0 + r < nrhs) B[pos + (size_t)(c0 + r) * ldb] = b[r];
        }
    }
}

// ---------------------------------------------------------------------------
// getrf
template <typename T, int NC, int NW>
__global__ void __launch_bounds__(32 * NW * BlockShape<NW>::MPB, MinBlocks<NC, NW>::value)
getrf_small_kernel(WorkList wl, LuSizes sz, T** dA_array, int** ipiv_array, int* info_array) {
    constexpr int MPB = BlockShape<NW>::MPB;
    __shared__ SmallLuShared<T, NC, NW> shm[MPB];
    const int local = (NW == 1) ? (threadIdx.x >> 5) : 0;
    const int tid = (NW == 1) ? (threadIdx.x & 31) : threadIdx.x;
    // NW == 1: each warp walks its own items; NW > 1: the block walks them together
    for (int w = blockIdx.x * MPB + local; w < wl.size(); w += gridDim.x * MPB) {
        getrf_small_instance<T, NC, NW>(wl.at(w), sz, dA_array, ipiv_array, info_array, tid, shm[local]);
        mat_sync<NW>();
    }
}

// ---------------------------------------------------------------------------
// gesv: getrf + getrs(NoTrans) in one pass. R = RHS columns solved together.
template <typename T, int NC, int NW, int R>
__global__ void __launch_bounds__(32 * NW * BlockShape<NW>::MPB, MinBlocks<NC, NW>::value)
gesv_small_kernel(WorkList wl, LuSizes sz, T** dA_array, int** ipiv_array, T** dB_array, int* info_array) {
    constexpr int MPB = BlockShape<NW>::MPB;
    __shared__ SmallLuShared<T, NC, NW> shm[MPB];
    const int local = (NW == 1) ? (threadIdx.x >> 5) : 0;
    const int tid = (NW == 1) ? (threadIdx.x & 31) : threadIdx.x;
    for (int w = blockIdx.x * MPB + local; w < wl.size(); w += gridDim.x * MPB) {
        gesv_small_instance<T, NC, NW, R>(wl.at(w), sz, dA_array, ipiv_array, dB_array, info_array, tid,
                                          shm[local]);
        mat_sync<NW>();
    }
}

// ---------------------------------------------------------------------------
// getrs, NoTrans. Thread tid loads LU row tid (already in final position) and
// moves b to P*b by replaying the ipiv swap sequence on indices.
template <typename T, int NC, int NW, int R>
__device__ __forceinline__ void permute_rhs(T (&b)[R], const int* ipiv, int n, int tid,
                                            SmallLuShared<T, NC, NW>& sh, T* xch, bool inverse) {
    static_assert(R <= 4, "the shared rhs buffer holds 4 right-hand sides a group");
    // idx = where the entry of original row tid sits after LAPACK's DLASWP
    // (forward: k ascending; inverse: k descending). No pivots: nothing moves.
    if (!ipiv) return;
    int idx = tid;
    if (!inverse) {
        for (int k = 0; k < n; ++k) {
            int p = ipiv[k] - 1;
            if (idx == k) idx = p; else if (idx == p) idx = k;
        }
    } else {
        for (int k = n - 1; k >= 0; --k) {
            int p = ipiv[k] - 1;
            if (idx == k) idx = p; else if (idx == p) idx = k;
        }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        if (tid < n) xch[idx] = b[r];
        mat_sync<NW>();
        if (tid < n) b[r] = xch[tid];
        mat_sync<NW>();
    }
}

template <typename T, int NC, int NW, int R, bool trans>
__global__ void __launch_bounds__(32 * NW * BlockShape<NW>::MPB, MinBlocks<NC, NW>::value)
getrs_small_kernel(WorkList wl, LuSizes sz, T** dA_array, int** ipiv_array, T** dB_array) {
    static_assert(R <= 4, "the shared rhs buffer holds 4 right-hand sides a group");
    constexpr int MPB = BlockShape<NW>::MPB;
    __shared__ SmallLuShared<T, NC, NW> shm[MPB];
    __shared__ T xch[MPB][32 * NW];
    const int local = (NW == 1) ? (threadIdx.x >> 5) : 0;
    const int tid = (NW == 1) ? (threadIdx.x & 31) : threadIdx.x;
    for (int w = blockIdx.x * MPB + local; w < wl.size(); w += gridDim.x * MPB) {
    const int id = wl.at(w);
    const int n = sz.get_n(id), lda = sz.get_lda(id), ldb = sz.get_ldb(id), nrhs = sz.get_nrhs(id);
    if (n <= 0 || nrhs <= 0) continue;
    const T* A = dA_array[id];
    T* B = dB_array[id];
    const int* ipiv = ipiv_array ? ipiv_array[id] : nullptr;   // null: factors without pivoting
    T a[NC];
    load_rows<T, NC, NW>(a, A, n, n, lda, tid);
    SmallLuShared<T, NC, NW>& sh = shm[local];
    const int pos = (tid < n) ? tid : INT_MAX / 2;
    for (int c0 = 0; c0 < nrhs; c0 += R) {
        T b[R];
#pragma unroll
        for (int r = 0; r < R; ++r) b[r] = (tid < n && c0 + r < nrhs) ? B[tid + (size_t)(c0 + r) * ldb] : T(0);
        if constexpr (!trans) {
            permute_rhs<T, NC, NW, R>(b, ipiv, n, tid, sh, xch[local], false);
            small_lu_solve<T, NC, NW, R>(a, n, pos, b, sh);
        } else {
            // A^T x = b:  U^T y = b (forward, non-unit), L^T z = y (backward, unit),
            // x = P^T z. Row k of U / L is published through shared memory.
            static_for<0, NC>([&](auto kc) {
                constexpr int k = decltype(kc)::value;
                if (k >= n) return;
                constexpr int buf = k & 1;
                if (tid == k) {
#pragma unroll
                    for (int r = 0; r < R; ++r) { b[r] = b[r] / a[k]; sh.rhs[buf][r] = b[r]; }
#pragma unroll
                    for (int j = k + 1; j < NC; ++j) sh.row[buf][j] = a[j];
                }
                mat_sync<NW>();
                if (tid > k && tid < n) {
                    const T u = sh.row[buf][tid];   // U(k, tid)
#pragma unroll
                    for (int r = 0; r < R; ++r) b[r] = fma_rn(-u, sh.rhs[buf][r], b[r]);
                }
            });
            static_for<0, NC>([&](auto ic) {
                constexpr int kk = NC - 1 - decltype(ic)::value;
                if (kk >= n) return;
                constexpr int buf = (kk + 1) & 1;
                if (tid == kk) {
#pragma unroll
                    for (int r = 0; r < R; ++r) sh.rhs[buf][r] = b[r];
#pragma unroll
                    for (int j = 0; j < kk; ++j) sh.row[buf][j] = a[j];
                }
                mat_sync<NW>();
                if (tid < kk) {
                    const T l = sh.row[buf][tid];   // L(kk, tid)
#pragma unroll
                    for (int r = 0; r < R; ++r) b[r] = fma_rn(-l, sh.rhs[buf][r], b[r]);
                }
            });
            permute_rhs<T, NC, NW, R>(b, ipiv, n, tid, sh, xch[local], true);
        }
        if (tid < n) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (c0 + r < nrhs) B[pos + (size_t)(c0 + r) * ldb] = b[r];
        }
        mat_sync<NW>();
    }
    }
}

// ---------------------------------------------------------------------------
// Launchers, explicitly instantiated per (NC, NW) in small_lu_inst_*.cu so the
// variants compile in parallel.
template <typename T, int NC, int NW>
void launch_getrf(const WorkList& wl, int grid, const LuSizes& sz, T** A, int** ipiv, int* info, cudaStream_t s) {
    constexpr int MPB = BlockShape<NW>::MPB;
    getrf_small_kernel<T, NC, NW><<<grid, 32 * NW * MPB, 0, s>>>(wl, sz, A, ipiv, info);
}

template <typename T, int NC, int NW>
void launch_gesv(const WorkList& wl, int grid, const LuSizes& sz, int max_nrhs, T** A, int** ipiv, T** B, int* info,
                 cudaStream_t s) {
    constexpr int MPB = BlockShape<NW>::MPB;
    if (max_nrhs <= 1)
        gesv_small_kernel<T, NC, NW, 1><<<grid, 32 * NW * MPB, 0, s>>>(wl, sz, A, ipiv, B, info);
    else
        gesv_small_kernel<T, NC, NW, 4><<<grid, 32 * NW * MPB, 0, s>>>(wl, sz, A, ipiv, B, info);
}

template <typename T, int NC, int NW>
void launch_getrs(const WorkList& wl, int grid, const LuSizes& sz, bool trans, int max_nrhs, T** A, int** ipiv, T** B,
                  cudaStream_t s) {
    constexpr int MPB = BlockShape<NW>::MPB;
    const dim3 block(32 * NW * MPB);
    if (trans) {
        if (max_nrhs <= 1) getrs_small_kernel<T, NC, NW, 1, true><<<grid, block, 0, s>>>(wl, sz, A, ipiv, B);
        else getrs_small_kernel<T, NC, NW, 4, true><<<grid, block, 0, s>>>(wl, sz, A, ipiv, B);
    } else {
        if (max_nrhs <= 1) getrs_small_kernel<T, NC, NW, 1, false><<<grid, block, 0, s>>>(wl, sz, A, ipiv, B);
        else getrs_small_kernel<T, NC, NW, 4, false><<<grid, block, 0, s>>>(wl, sz, A, ipiv, B);
    }
}

#define MB200_INSTANTIATE_SMALL(T, NC, NW)                                                                   \
    template void launch_getrf<T, NC, NW>(const WorkList&, int, const LuSizes&, T**, int**, int*, cudaStream_t); \
    template void launch_gesv<T, NC, NW>(const WorkList&, int, const LuSizes&, int, T**, int**, T**, int*,       \
                                         cudaStream_t);                                                          \
    template void launch_getrs<T, NC, NW>(const WorkList&, int, const LuSizes&, bool, int, T**, int**, T**,      \
                                          cudaStream_t);

}  // namespace mb200

// Every (type, column bound, warps per matrix) the dispatcher may select.
#define MB200_SMALL_VARIANTS(X) \
    X(double, 8, 1) X(double, 16, 1) X(double, 32, 1) X(double, 64, 1) \
    X(double, 32, 2) X(double, 64, 2) X(double, 32, 4) X(double, 64, 4) \
    X(float, 8, 1) X(float, 16, 1) X(float, 32, 1) X(float, 64, 1) \
    X(float, 32, 2) X(float, 64, 2) X(float, 32, 4) X(float, 64, 4)
