// qr.cu -- batched Householder QR (magma_dgeqrf_batched, src/zgeqrf_batched.cpp:89-230).
//
// LAPACK dgeqr2 order: for each column k, dlarfg on A(k:m, k), then dlarf on the
// trailing columns. One thread block per matrix; P consecutive lanes per column
// (P = 1, 2, 4, 8 for m <= 16, 32, 64, 128; P = 8 with 32 rows a lane for m <= 256,
// with 64 rows a lane for m <= 512; P = 16 with 64 rows a lane for m <= 1024);
// lane p of column j holds rows r = i*P + p (i < S) in registers, so a warp's
// load or store of element i touches P consecutive rows of each of its columns
// (sector-coalesced without staging). Rows >= m are zero.
//
// More columns than a panel holds (64; 32 for m > 256, 16 for m > 512): the columns are processed in panels (one panel's
// columns in registers); a panel first replays, in order, the reflectors the
// earlier panels formed (read back from A and tau), then forms its own. Every
// column receives the same operations in the same order either way.
//
// Step k (one barrier; the shared vectors are double-buffered by step parity):
//   the P lanes of column k:  xs_p = sum_{r>k, r=p mod P} a_r^2 (ascending fma chain),
//     xs = pairwise tree over p, beta = -sign(alpha) sqrt(fma(alpha, alpha, xs)),
//     tau = (beta - alpha) / beta, scal = 1 / (alpha - beta), v_r = a_r * scal;
//     publish sv_r = (0 for r < k, 1 for r = k, v_r for r > k) and stv_r = -tau * sv_r;
//   every column j > k:  w_p = sum over its rows of sv_r a_r (ascending fma chain from 0),
//     w = pairwise tree over p, a_r = fma(stv_r, w, a_r) for all its rows.
// The oracle restates exactly this order (rows above k enter with zero weights), so
// the factors are BIT-IDENTICAL to it; against LAPACK dgeqrf they agree to rounding.
// tau = 0 when xs == 0 (H = I). Without dnrm2's scaling and dlapy2's guard, entries
// must lie well inside [1e-150, 1e150] (far beyond the inputs this path serves).
#include "internal.h"
#include "small_lu.cuh"
#include <algorithm>

namespace mb200 {

// Sum over the P lanes of a column group (xor butterfly = pairwise tree in lane order;
// every lane ends with the same value since IEEE addition commutes).
template <int P>
__device__ __forceinline__ double group_sum(double x, unsigned mask) {
#pragma unroll
    for (int o = 1; o < P; o <<= 1) x += __shfl_xor_sync(mask, x, o);
    return x;
}

// Register budget: 64 a thread for S = 16, 128 for S = 32 and 255 for S = 64 (the S
// entries of a plus the shared vectors' pairs in flight).
template <int S, int P, int NCOL>
__global__ void __launch_bounds__(P * NCOL, (S == 16 ? 1024 : S == 32 ? 512 : 256) / (P * NCOL) < 1 ? 1
                                            : (S == 16 ? 1024 : S == 32 ? 512 : 256) / (P * NCOL))
geqrf_lanes_kernel(int m, int n, double** dA_array, int lda, double** dtau_array, int batch) {
    constexpr int SP = S + 2;   // padded, even lane stride in the shared vectors
    static_assert(S % 2 == 0 && 32 % P == 0, "layout");
    __shared__ __align__(16) double sv[2][P * SP];
    __shared__ __align__(16) double stv[2][P * SP];
    __shared__ double stau[2];
    const int tid = threadIdx.x, lane = tid & 31, p = tid % P, j = tid / P;
    constexpr int CPW = 32 / P;                               // columns per warp
    const int wc0 = (tid >> 5) * CPW;                         // the warp's first column
    const unsigned gmask = P == 32 ? 0xffffffffu : (((1u << P) - 1) << (lane & ~(P - 1)));
    const int kmax = min(m, n);
    // Publishes reflector k (column k of A0 below the diagonal, tau[k]) in the shared
    // vectors of buffer b: sv_r = 0 (r < k), 1 (r = k), v_r (r > k), stv_r = -tau sv_r --
    // the values the step that formed it published.
    auto stage_reflector = [&](const double* A0, int k, double t, int b) {
        for (int idx = tid; idx < P * S; idx += P * NCOL) {
            const int pp = idx % P, i = idx / P, r = i * P + pp;
            const double v = r > k ? (r < m ? A0[r + (size_t)k * lda] : 0.0) : (r == k ? 1.0 : 0.0);
            sv[b][pp * SP + i] = v;
            stv[b][pp * SP + i] = -t * v;
        }
        if (tid == 0) stau[b] = t;
    };
    // Column col (this thread's) takes reflector k from buffer b, if col is in (k, n).
    auto apply_reflector = [&](double (&a)[S], int k, int b, int col, int c0) {
        const double t = stau[b];
        if (t != 0.0 && c0 + wc0 + CPW - 1 > k && c0 + wc0 < n) {   // the warp has a column in (k, n)
            const double* svp = sv[b] + p * SP;
            const double* stp = stv[b] + p * SP;
            double w = 0.0;
#pragma unroll
            for (int i = 0; i < S; i += 2) {
                const double2 v = *reinterpret_cast<const double2*>(svp + i);
                w = fma(v.x, a[i], w);
                w = fma(v.y, a[i + 1], w);
            }
            w = group_sum<P>(w, 0xffffffffu);
            if (col > k && col < n) {
#pragma unroll
                for (int i = 0; i < S; i += 2) {
                    const double2 tv = *reinterpret_cast<const double2*>(stp + i);
                    a[i] = fma(tv.x, w, a[i]);
                    a[i + 1] = fma(tv.y, w, a[i + 1]);
                }
            }
        }
    };
    for (int id = blockIdx.x; id < batch; id += gridDim.x) {
        double* A0 = dA_array[id];
        double* tau = dtau_array[id];
        // columns in panels of NCOL: a panel first takes, in order, the reflectors of the
        // panels before it (read back from A and tau), then forms its own -- every column
        // receives the same operations in the same order as in the unblocked algorithm
        for (int c0 = 0; c0 < n; c0 += NCOL) {
            const int col = c0 + j;
            double* A = A0 + (size_t)col * lda;
            double a[S];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const int r = i * P + p;
                a[i] = (col < n && r < m) ? A[r] : 0.0;
            }
#pragma unroll 1
            for (int k = 0; k < min(c0, kmax); ++k) {
                const int b = k & 1;
                stage_reflector(A0, k, tau[k], b);
                __syncthreads();
                apply_reflector(a, k, b, col, c0);
            }
#pragma unroll 1
            for (int k = c0; k < min(kmax, c0 + NCOL); ++k) {
                const int b = k & 1;
                if (col == k) {
                    // branch-free: rows <= k enter the chain as fma(a, 0, xs) = xs exactly (xs >= +0)
                    double xs = 0.0, al = 0.0;
#pragma unroll
                    for (int i = 0; i < S; ++i) {
                        const int r = i * P + p;
                        xs = fma(a[i], r > k ? a[i] : 0.0, xs);
                        al = r == k ? a[i] : al;
                    }
                    xs = group_sum<P>(xs, gmask);
                    const double alpha = P == 1 ? al : __shfl_sync(gmask, al, (lane & ~(P - 1)) | (k % P));
                    double t = 0.0, beta = alpha, scal = 1.0;
                    if (xs > 0.0) {
                        beta = -copysign(sqrt(fma(alpha, alpha, xs)), alpha);
                        t = (beta - alpha) / beta;
                        scal = 1.0 / (alpha - beta);
                    }
                    double* svp = sv[b] + p * SP;
                    double* stp = stv[b] + p * SP;
                    const bool scaled = t != 0.0;
#pragma unroll
                    for (int i = 0; i < S; i += 2) {
                        double v2[2];
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int r = (i + h) * P + p;
                            const double x = a[i + h] * scal;
                            v2[h] = r > k ? x : (r == k ? 1.0 : 0.0);
                            a[i + h] = (r > k && scaled) ? x : (r == k ? beta : a[i + h]);
                        }
                        *reinterpret_cast<double2*>(svp + i) = make_double2(v2[0], v2[1]);
                        *reinterpret_cast<double2*>(stp + i) = make_double2(-t * v2[0], -t * v2[1]);
                    }
                    if (p == 0) {
                        stau[b] = t;
                        tau[k] = t;
                    }
                }
                __syncthreads();
                apply_reflector(a, k, b, col, c0);
            }
            if (col < n) {
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    const int r = i * P + p;
                    if (r < m) A[r] = a[i];
                }
            }
            __syncthreads();   // the panel's columns and tau are in memory before the next panel reads them
        }
    }
}

template <int S, int P>
static void launch_geqrf(int m, int n, double** A, int lda, double** tau, int batch, cudaStream_t s) {
    const int grid = std::min(batch, 65535);
    if constexpr (P == 16) {   // 256 threads
        geqrf_lanes_kernel<S, P, 16><<<grid, P * 16, 0, s>>>(m, n, A, lda, tau, batch);
    } else {
        if (n <= 16 && P * 16 >= 32 && S <= 32) geqrf_lanes_kernel<S, P, 16><<<grid, P * 16, 0, s>>>(m, n, A, lda, tau, batch);
        else if (n <= 32 || S > 32) geqrf_lanes_kernel<S, P, 32><<<grid, P * 32, 0, s>>>(m, n, A, lda, tau, batch);
        else geqrf_lanes_kernel<S, P, 64><<<grid, P * 64, 0, s>>>(m, n, A, lda, tau, batch);
    }
}

bool geqrf_supported(int m, int n) { return m <= 1024 && n >= 0; }

magma_int_t geqrf_small(int m, int n, double** A, int lda, double** tau, int batch, cudaStream_t s) {
    if (!geqrf_supported(m, n)) return MAGMA_ERR_NOT_SUPPORTED;
    if (m <= 16) launch_geqrf<16, 1>(m, n, A, lda, tau, batch, s);
    else if (m <= 32) launch_geqrf<16, 2>(m, n, A, lda, tau, batch, s);
    else if (m <= 64) launch_geqrf<16, 4>(m, n, A, lda, tau, batch, s);
    else if (m <= 128) launch_geqrf<16, 8>(m, n, A, lda, tau, batch, s);
    else if (m <= 256) launch_geqrf<32, 8>(m, n, A, lda, tau, batch, s);
    else if (m <= 512) launch_geqrf<64, 8>(m, n, A, lda, tau, batch, s);   // panels of 32 columns, 64 rows a lane
    else launch_geqrf<64, 16>(m, n, A, lda, tau, batch, s);                // panels of 16 columns, 64 rows a lane
    return launch_status();
}

}  // namespace mb200

using namespace mb200;

extern "C" {

// src/zgeqrf_batched.cpp:89-119: info_array zeroed first; m -1, n -2, ldda < max(1,m) -4;
// quick return when m or n is 0. m <= 1024 (MAGMA_ERR_NOT_SUPPORTED otherwise), any n.
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
