// getri.cu -- batched out-of-place inverse from the LU factors
// (magma_dgetri_outofplace_batched, src/zgetri_outofplace_batched.cpp:82-220).
//
// The reference sets inv(A) = I, solves U^-1 L^-1 I with two out-of-place batched
// trsm's (trtri-based diagonal blocks) and then applies the column interchanges of
// ipiv in reverse order. Here inv(A) = I, then the batched getrs kernels solve
// A X = I in place with the row interchanges applied to I first: every column of
// the result is the solve of one unit vector, so the columns are the reference's
// U^-1 L^-1 e_i, moved to their interchanged positions (for n <= 32 one fused kernel,
// getri_small_kernel, does the same operations). info_array receives the
// 1-based index of the first exactly-zero diagonal entry of U (0 when none), the
// condition the reference documents for its info.
#include "internal.h"
#include "batched_kernels.h"
#include <algorithm>

namespace mb200 {

// One block per instance: invA = I, info = first zero on the diagonal of U.
__global__ void getri_setup_kernel(int n, double** dA_array, int ldda, double** dinvA_array, int lddia,
                                   int* info_array, int batch) {
    for (int id = blockIdx.x; id < batch; id += gridDim.x) {
        double* W = dinvA_array[id];
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int i = idx % n, j = idx / n;
            W[i + (size_t)j * lddia] = (i == j) ? 1.0 : 0.0;
        }
        if (info_array) {
            const double* A = dA_array[id];
            int first = n + 1;
            for (int i = threadIdx.x; i < n; i += blockDim.x)
                if (A[i + (size_t)i * ldda] == 0.0) first = min(first, i + 1);
            for (int off = 16; off > 0; off >>= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, off));
            __shared__ int red[32];
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = first;
            __syncthreads();
            if (threadIdx.x == 0) {
                int m = n + 1;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = min(m, red[w]);
                info_array[id] = (m == n + 1) ? 0 : m;
            }
            __syncthreads();
        }
    }
}

// n <= 32: one warp per matrix, lane c computes column c of inv(A) with the whole
// column in registers and the LU factors in shared memory (broadcast reads). The
// operations are the oracle's dgetrs on B = I, in its order: the row interchanges
// applied to e_c (tracked as the position of its single 1), then
//   for k ascending, i > k:   x_i = fma(-x_k, L(i,k), x_i)
//   for k descending:         x_k = x_k / U(k,k);  i < k: x_i = fma(-x_k, U(i,k), x_i)
// so the result is bit-identical to the getrs path (and to the oracle). Rows and
// columns past n are padded with the identity: their terms add -0, which leaves
// every value unchanged. The columns are staged back through shared memory so the
// stores coalesce; info = first zero on U's diagonal, from a warp ballot.
constexpr int kGetriWarps = 4;

__global__ void __launch_bounds__(32 * kGetriWarps)
getri_small_kernel(int n, double** dA_array, int ldda, int** dipiv_array, double** dinvA_array, int lddia,
                   int* info_array, int batch) {
    __shared__ double sLU[kGetriWarps][32][33];   // [warp][column][row]
    __shared__ int sP[kGetriWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double (*L)[33] = sLU[w];
    for (int id = blockIdx.x * kGetriWarps + w; id < batch; id += gridDim.x * kGetriWarps) {
        const double* A = dA_array[id];
        for (int j = 0; j < 32; ++j) L[j][lane] = (j < n && lane < n) ? A[lane + (size_t)j * ldda]
                                                                      : (lane == j ? 1.0 : 0.0);
        sP[w][lane] = lane < n ? dipiv_array[id][lane] - 1 : lane;
        __syncwarp();
        int pos = lane;
        for (int k = 0; k < n; ++k) {
            const int p = sP[w][k];
            pos = (pos == k) ? p : (pos == p ? k : pos);
        }
        double x[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) x[i] = (i == pos) ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            const double xk = x[k];
#pragma unroll
            for (int i = k + 1; i < 32; ++i) x[i] = fma(-xk, L[k][i], x[i]);
        }
#pragma unroll
        for (int k = 31; k >= 0; --k) {
            x[k] = x[k] / L[k][k];
            const double xk = x[k];
#pragma unroll
            for (int i = 0; i < k; ++i) x[i] = fma(-xk, L[k][i], x[i]);
        }
        const unsigned zero = __ballot_sync(0xffffffffu, lane < n && L[lane][lane] == 0.0);
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 32; ++i) L[lane][i] = x[i];   // column `lane` of inv(A)
        __syncwarp();
        double* W = dinvA_array[id];
        for (int j = 0; j < n; ++j)
            if (lane < n) W[lane + (size_t)j * lddia] = L[j][lane];
        if (info_array && lane == 0) info_array[id] = zero ? __ffs(zero) : 0;
        __syncwarp();
    }
}

}  // namespace mb200

using namespace mb200;

extern "C" {

// src/zgetri_outofplace_batched.cpp:89-105: n -> -1, ldda < max(1,n) -> -3,
// lddia < max(1,n) -> -6; quick return when n == 0.
magma_int_t magma_dgetri_outofplace_batched(magma_int_t n, double** dA_array, magma_int_t ldda,
                                            magma_int_t** dipiv_array, double** dinvA_array, magma_int_t lddia,
                                            magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t info = 0;
    if (n < 0) info = -1;
    else if (ldda < std::max(1, n)) info = -3;
    else if (lddia < std::max(1, n)) info = -6;
    if (info != 0) {
        magma_xerbla(__func__, -info);
        return info;
    }
    if (n == 0 || batchCount <= 0) return 0;
    if (!small_lu_supported(n, n) && !blocked_lu_supported(n)) return MAGMA_ERR_NOT_SUPPORTED;
    if (n <= 32) {
        const int grid = std::min(ceildiv(batchCount, kGetriWarps), 65535);
        getri_small_kernel<<<grid, 32 * kGetriWarps, 0, queue->stream>>>(n, dA_array, ldda, dipiv_array,
                                                                        dinvA_array, lddia, info_array, batchCount);
        return launch_status();
    }
    getri_setup_kernel<<<std::min(batchCount, 4096), 256, 0, queue->stream>>>(n, dA_array, ldda, dinvA_array,
                                                                               lddia, info_array, batchCount);
    const WorkList wl{nullptr, nullptr, batchCount};
    const LuSizes sz{n, n, ldda, lddia, n, nullptr, nullptr, nullptr, nullptr, nullptr};
    magma_int_t rc = small_lu_supported(n, n)
                         ? getrs_small<double>(wl, batchCount, false, false, sz, n, n, dA_array, dipiv_array,
                                               dinvA_array, queue->stream)
                         : getrs_blocked<double>(wl, batchCount, false, false, sz, n, n, dA_array, dipiv_array,
                                                 dinvA_array, queue->stream);
    return rc ? rc : launch_status();
}

}  // extern "C"
