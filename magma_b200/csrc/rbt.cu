// rbt.cu -- random butterfly transformation and the batched RBT solve
// (magma_dgerbt_batched, src/zgerbt_batched.cpp:118-190; magma_dgesv_rbt_batched,
// src/zgesv_rbt_batched.cpp:81-170).
//
// A depth-2 partial random butterfly W = L2 L1 of order n (n a multiple of 4):
//   L1, the order-n butterfly with diagonal weights r = w[0..n-1]:
//     (L1 x)_i = (r_i x_i + r_{h+i} x_{h+i}) / sqrt2,  (L1 x)_{h+i} = (r_i x_i - r_{h+i} x_{h+i}) / sqrt2,
//     i < h = n/2;
//   L2, two order-h butterflies on the halves with weights s = w[n..2n-1].
// With U and V built from the caller's vectors u and v (2n entries each), the
// system is transformed to (U^T A V) y = U^T b, factored without pivoting, and
// x = V y. The randomisation makes pivoting unnecessary with high probability
// (Parker's RBT). gen = true fills u and v like the reference (exp((t - 1/2)/10),
// t uniform on [0,1)), here from a fixed-seed splitmix64 stream instead of the
// C library's rand(), so the transform is reproducible.
#include "internal.h"
#include "batched_kernels.h"
#include <algorithm>
#include <cmath>
#include <vector>

namespace mb200 {

// One butterfly level on the entries (i, i + half) of every pair inside blocks of 2*half:
// transposed form  x_i' = w_i (x_i + x_p) / sqrt2,  x_p' = w_p (x_i - x_p) / sqrt2
// forward form     x_i' = (w_i x_i + w_p x_p) / sqrt2,  x_p' = (w_i x_i - w_p x_p) / sqrt2
__device__ __forceinline__ void butterfly_pair(double& xi, double& xp, double wi, double wp, bool transposed) {
    const double c = 0.70710678118654752440;   // 1/sqrt(2)
    const double a = xi, b = xp;
    if (transposed) {
        xi = wi * (a + b) * c;
        xp = wp * (a - b) * c;
    } else {
        xi = (wi * a + wp * b) * c;
        xp = (wi * a - wp * b) * c;
    }
}

// Applies one level (block size 2*half, weights w) along dimension `rows`
// (true: to every column vector of the n x ncols matrix M; false: combining
// columns, i.e. to every row vector of the n x n matrix M), in the transposed form.
__device__ void level_on_matrix(double* M, int ld, int n, int ncols, int half, const double* w, bool along_rows) {
    const int pairs = n / 2;
    if (along_rows) {
        for (int idx = threadIdx.x; idx < pairs * ncols; idx += blockDim.x) {
            const int q = idx % pairs, c = idx / pairs;
            const int i = (q / half) * 2 * half + q % half, p = i + half;
            butterfly_pair(M[i + (size_t)c * ld], M[p + (size_t)c * ld], w[i], w[p], true);
        }
    } else {
        for (int idx = threadIdx.x; idx < pairs * n; idx += blockDim.x) {
            const int r = idx % n, q = idx / n;
            const int i = (q / half) * 2 * half + q % half, p = i + half;
            butterfly_pair(M[r + (size_t)i * ld], M[r + (size_t)p * ld], w[i], w[p], true);
        }
    }
}

// A <- U^T A V for each instance, one block per instance.
__global__ void rbt_matrix_kernel(int n, double** dA_array, int lda, const double* u, const double* v, int batch) {
    for (int id = blockIdx.x; id < batch; id += gridDim.x) {
        double* A = dA_array[id];
        level_on_matrix(A, lda, n, n, n / 4, u + n, true);   // U^T = L1^T L2^T: L2^T first
        __syncthreads();
        level_on_matrix(A, lda, n, n, n / 2, u, true);
        __syncthreads();
        level_on_matrix(A, lda, n, n, n / 4, v + n, false);  // V = L2 L1: A L2 first
        __syncthreads();
        level_on_matrix(A, lda, n, n, n / 2, v, false);
        __syncthreads();
    }
}

// B <- U^T B (transpose form) or B <- V B (forward form: L1 first, then L2).
__global__ void rbt_rhs_kernel(int n, int nrhs, double** dB_array, int ldb, const double* w, bool transposed,
                               int batch) {
    for (int id = blockIdx.x; id < batch; id += gridDim.x) {
        double* B = dB_array[id];
        const int pairs = n / 2;
        for (int level = 0; level < 2; ++level) {
            // transposed: L2^T then L1^T; forward: L1 then L2
            const bool full = transposed ? (level == 1) : (level == 0);
            const int half = full ? n / 2 : n / 4;
            const double* wl = full ? w : w + n;
            for (int idx = threadIdx.x; idx < pairs * nrhs; idx += blockDim.x) {
                const int q = idx % pairs, c = idx / pairs;
                const int i = (q / half) * 2 * half + q % half, p = i + half;
                butterfly_pair(B[i + (size_t)c * ldb], B[p + (size_t)c * ldb], wl[i], wl[p], transposed);
            }
            __syncthreads();
        }
    }
}

static void init_butterfly(int count, double* w, unsigned long long seed) {
    unsigned long long x = seed;
    for (int i = 0; i < count; ++i) {
        unsigned long long z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        const double t = double(z >> 11) * (1.0 / 9007199254740992.0);
        w[i] = std::exp((t - 0.5) / 10.0);
    }
}

}  // namespace mb200

using namespace mb200;

extern "C" {

// src/zgerbt_batched.cpp:118-190: gen -1, n -2, nrhs -3, ldda -5, lddb -7 (written to
// *info and returned). U and V are host vectors of 2n entries (filled when gen is true).
magma_int_t magma_dgerbt_batched(magma_bool_t gen, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                 magma_int_t ldda, double** dB_array, magma_int_t lddb, double* U, double* V,
                                 magma_int_t* info, magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t arg = 0;
    if (gen != MagmaTrue && gen != MagmaFalse) arg = -1;
    else if (n < 0) arg = -2;
    else if (nrhs < 0) arg = -3;
    else if (ldda < std::max(1, n)) arg = -5;
    else if (lddb < std::max(1, n)) arg = -7;
    if (info) *info = arg;
    if (arg != 0) {
        magma_xerbla(__func__, -arg);
        return arg;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    if (n % 4 != 0) return MAGMA_ERR_NOT_SUPPORTED;
    if (gen == MagmaTrue) {
        init_butterfly(2 * n, U, 0x5EEDull);
        init_butterfly(2 * n, V, 0xB0B5EEDull);
    }
    double* d = static_cast<double*>(queue_workspace(queue, sizeof(double) * 4 * n));
    if (!d) return MAGMA_ERR_DEVICE_ALLOC;
    cudaMemcpyAsync(d, U, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, queue->stream);
    cudaMemcpyAsync(d + 2 * n, V, sizeof(double) * 2 * n, cudaMemcpyHostToDevice, queue->stream);
    const int grid = std::min(batchCount, 4096);
    rbt_matrix_kernel<<<grid, 256, 0, queue->stream>>>(n, dA_array, ldda, d, d + 2 * n, batchCount);
    rbt_rhs_kernel<<<grid, 256, 0, queue->stream>>>(n, nrhs, dB_array, lddb, d, true, batchCount);
    // (copies from pageable host memory return once the vectors are staged: U and V may be reused)
    return launch_status();
}

// src/zgesv_rbt_batched.cpp:81-170: n -1, nrhs -2, ldda -4, lddb -6. Transform with a
// fresh butterfly, LU without pivoting, solve, x = V y. n a multiple of 4, <= 1024.
magma_int_t magma_dgesv_rbt_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                    double** dB_array, magma_int_t lddb, magma_int_t* dinfo_array,
                                    magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t info = 0;
    if (n < 0) info = -1;
    else if (nrhs < 0) info = -2;
    else if (ldda < std::max(1, n)) info = -4;
    else if (lddb < std::max(1, n)) info = -6;
    if (info != 0) {
        magma_xerbla(__func__, -info);
        return info;
    }
    if (n == 0 || nrhs == 0 || batchCount <= 0) return 0;
    if (n % 4 != 0 || (!small_lu_supported(n, n) && !blocked_lu_supported(n))) return MAGMA_ERR_NOT_SUPPORTED;
    std::vector<double> hu(2 * n), hv(2 * n);
    magma_int_t arg = 0;
    magma_int_t rc = magma_dgerbt_batched(MagmaTrue, n, nrhs, dA_array, ldda, dB_array, lddb, hu.data(), hv.data(),
                                          &arg, batchCount, queue);
    if (rc) return rc;
    rc = magma_dgetrf_nopiv_batched(n, n, dA_array, ldda, dinfo_array, batchCount, queue);
    if (rc) return rc;
    rc = magma_dgetrs_nopiv_batched(MagmaNoTrans, n, nrhs, dA_array, ldda, dB_array, lddb, nullptr, batchCount,
                                    queue);
    if (rc) return rc;
    // x = V y with V's vectors still in the queue workspace (the second 2n entries)
    const double* d = static_cast<const double*>(queue_workspace(queue, sizeof(double) * 4 * n));
    rbt_rhs_kernel<<<std::min(batchCount, 4096), 256, 0, queue->stream>>>(n, nrhs, dB_array, lddb, d + 2 * n, false,
                                                                         batchCount);
    return launch_status();
}

}  // extern "C"
