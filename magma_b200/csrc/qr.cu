// qr.cu -- batched Householder QR (magma_dgeqrf_batched, src/zgeqrf_batched.cpp:89-230).
//
// One thread block per matrix, thread t = row t, the row's n <= NC entries in
// registers (the register-resident layout of the LU kernels). For each column k
// (LAPACK dgeqr2 order: dlarfg, then dlarf on the trailing columns):
//   xnorm = ||A(k+1:m, k)|| by a block reduction, beta = -sign(alpha) hypot(alpha, xnorm),
//   tau = (beta - alpha) / beta, v = A(k+1:m, k) / (alpha - beta), A(k,k) = beta
//   (tau = 0 when xnorm == 0: H = I);
//   w = v^T A(k:m, k+1:n) for all trailing columns at once: every thread forms
//   v_t A(t, j), each warp reduces its 32 rows for 32 columns with one reduce-scatter
//   of 31 shuffles (lane j ends with column j's sum), warps are combined in shared
//   memory;  A(k:m, k+1:n) -= tau v w^T.
// The factors use LAPACK's representation: R on and above the diagonal, the
// Householder vectors (unit leading entry implied) below it, tau per reflector.
// Unlike LAPACK's dlarfg there is no rescaling loop for |beta| < safmin (orders of
// magnitude below the inputs this path serves); the sums run in tree order, so
// results agree with LAPACK to rounding, not bit for bit.
#include "internal.h"
#include "small_lu.cuh"
#include <algorithm>

namespace mb200 {

template <int NC, int NT>
struct QrShared {
    double red[NT / 32][NC];   // per-warp column sums
    double w[NC];              // v^T A for the trailing columns
    double col[NT / 32];       // per-warp partial of ||x||^2
    double alpha;
};

// Lane l of the warp returns sum over lanes of v[l] (columns base..base+31 of `v`).
__device__ __forceinline__ double warp_reduce_scatter32(double (&v)[32], int lane) {
    static_for<0, 5>([&](auto sc) {
        constexpr int s = 16 >> decltype(sc)::value;
        const bool upper = (lane & s) != 0;
#pragma unroll
        for (int i = 0; i < s; ++i) {
            const double send = upper ? v[i] : v[i + s];
            const double keep = upper ? v[i + s] : v[i];
            v[i] = keep + __shfl_xor_sync(kFullMask, send, s);
        }
    });
    return v[0];
}

template <int NC, int NT>
__global__ void __launch_bounds__(NT)
geqrf_small_kernel(int m, int n, double** dA_array, int lda, double** dtau_array, int batch) {
    constexpr int NW = NT / 32;
    __shared__ QrShared<NC, NT> sh;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int kmax = min(m, n);
    for (int id = blockIdx.x; id < batch; id += gridDim.x) {
        double* A = dA_array[id];
        double* tau = dtau_array[id];
        double a[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) a[j] = (t < m && j < n) ? A[t + (size_t)j * lda] : 0.0;
        static_for<0, NC>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            if (k >= kmax) return;
            // ---- dlarfg on A(k:m, k) ----
            double xs = (t > k && t < m) ? a[k] * a[k] : 0.0;
            for (int off = 16; off > 0; off >>= 1) xs += __shfl_xor_sync(kFullMask, xs, off);
            if (lane == 0) sh.col[warp] = xs;
            if (t == k) sh.alpha = a[k];
            __syncthreads();
            double xnorm2 = 0.0;
#pragma unroll
            for (int w = 0; w < NW; ++w) xnorm2 += sh.col[w];
            const double alpha = sh.alpha;
            double tk = 0.0, scal = 0.0, beta = alpha;
            if (xnorm2 > 0.0) {
                beta = -copysign(hypot(alpha, sqrt(xnorm2)), alpha);
                tk = (beta - alpha) / beta;
                scal = 1.0 / (alpha - beta);
            }
            // v: 1 at row k, scaled entries below, 0 above
            const double v = (t == k) ? 1.0 : ((t > k && t < m) ? a[k] * scal : 0.0);
            if (t > k && t < m && xnorm2 > 0.0) a[k] = v;
            if (t == k) {
                a[k] = beta;
                tau[k] = tk;
            }
            // ---- w = v^T A(k:m, k+1:n), then A -= tau v w^T ----
            if (k + 1 < n) {
                constexpr int G0 = ((k + 1) / 32) * 32;   // first 32-column group with trailing columns
                static_for<G0 / 32, NC / 32>([&](auto gc) {
                    constexpr int g0 = decltype(gc)::value * 32;
                    double p[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) p[j] = (g0 + j > k) ? v * a[g0 + j] : 0.0;
                    const double s = warp_reduce_scatter32(p, lane);
                    sh.red[warp][g0 + lane] = s;
                });
                __syncthreads();
                if (t < NC && t > k) {
                    double s = 0.0;
#pragma unroll
                    for (int w = 0; w < NW; ++w) s += sh.red[w][t];
                    sh.w[t] = s;
                }
                __syncthreads();
                if (v != 0.0 && tk != 0.0) {
                    const double tv = tk * v;
#pragma unroll
                    for (int j = k + 1; j < NC; ++j) a[j] = fma(-tv, sh.w[j], a[j]);
                }
            }
            __syncthreads();
        });
        if (t < m) {
#pragma unroll
            for (int j = 0; j < NC; ++j)
                if (j < n) A[t + (size_t)j * lda] = a[j];
        }
        __syncthreads();
    }
}

template <int NC, int NT>
static void launch_geqrf(int m, int n, double** A, int lda, double** tau, int batch, cudaStream_t s) {
    geqrf_small_kernel<NC, NT><<<std::min(batch, 65535), NT, 0, s>>>(m, n, A, lda, tau, batch);
}

bool geqrf_supported(int m, int n) { return m <= 256 && n <= 64; }

magma_int_t geqrf_small(int m, int n, double** A, int lda, double** tau, int batch, cudaStream_t s) {
    if (!geqrf_supported(m, n)) return MAGMA_ERR_NOT_SUPPORTED;
    const int NT = m <= 32 ? 32 : m <= 64 ? 64 : m <= 128 ? 128 : 256;
    if (n <= 32) {
        if (NT == 32) launch_geqrf<32, 32>(m, n, A, lda, tau, batch, s);
        else if (NT == 64) launch_geqrf<32, 64>(m, n, A, lda, tau, batch, s);
        else if (NT == 128) launch_geqrf<32, 128>(m, n, A, lda, tau, batch, s);
        else launch_geqrf<32, 256>(m, n, A, lda, tau, batch, s);
    } else {
        if (NT <= 64) launch_geqrf<64, 64>(m, n, A, lda, tau, batch, s);
        else if (NT == 128) launch_geqrf<64, 128>(m, n, A, lda, tau, batch, s);
        else launch_geqrf<64, 256>(m, n, A, lda, tau, batch, s);
    }
    return launch_status();
}

}  // namespace mb200

using namespace mb200;

extern "C" {

// src/zgeqrf_batched.cpp:89-119: info_array zeroed first; m -1, n -2, ldda < max(1,m) -4;
// quick return when m or n is 0. m <= 256, n <= 64 (MAGMA_ERR_NOT_SUPPORTED otherwise).
magma_int_t magma_dgeqrf_batched(magma_int_t m, magma_int_t n, double** dA_array, magma_int_t ldda,
                                 double** dtau_array, magma_int_t* info_array, magma_int_t batchCount,
                                 magma_queue_t queue) {
    if (info_array && batchCount > 0) cudaMemsetAsync(info_array, 0, sizeof(magma_int_t) * batchCount, queue->stream);
    magma_int_t arginfo = 0;
    if (m < 0) arginfo = -1;
    else if (n < 0) arginfo = -2;
    else if (ldda < std::max(1, m)) arginfo = -4;
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    if (m == 0 || n == 0 || batchCount <= 0) return 0;
    return geqrf_small(m, n, dA_array, ldda, dtau_array, batchCount, queue->stream);
}

}  // extern "C"
