// small_lu.cuh -- register-resident LU factorisation and triangular solves
// for matrices with at most 32*NW rows and NC <= 64 columns.
//
// Layout: one thread owns one row of the matrix for the whole factorisation
// (NC values in registers). Rows are never moved between threads. Instead each
// thread tracks `pos`, the row position its row currently has in LAPACK's
// physically-swapped matrix: choosing the pivot of step k swaps the `pos` of
// the pivot row and of the row sitting at position k, exactly mirroring
// DSWAP in LAPACK's dgetf2, and at the end a thread stores its row at `pos`.
// This removes the row-swap traffic of the reference (zswap_kernel_batched,
// magmablas/zgetf2_kernels.cu:354; zlaswp_rowparallel, zlaswp_batched.cu:81).
//
// Arithmetic order is that of LAPACK's unblocked dgetf2 + reference BLAS
// (the algorithm MAGMA's testers check against, testing_zgetrf_batched.cpp:200):
//   pivot  = first row position with the largest |a(i,k)| (IDAMAX: ties go to
//            the lowest position),
//   scale  = multiply by the correctly rounded 1/pivot when |pivot| >= DBL_MIN,
//            else divide (dgetf2's SFMIN branch),
//   update = a(i,j) = fma(l(i), -u(j), a(i,j))  (DGER, one rank-1 step at a time).
// With these rules the factors, pivots and info are bit-identical to the
// project's CPU restatement of dgetf2 (oracle/), which is how the tests check
// them. The pivot-row broadcast goes through shared memory (double-buffered by
// step parity, so one barrier per step suffices).
#pragma once

#include <cuda_runtime.h>
#include <cfloat>
#include <climits>
#include <type_traits>

namespace mb200 {

constexpr unsigned kFullMask = 0xffffffffu;

// Compile-time loop: calls f(std::integral_constant<int, I>) for I in [Begin, End).
// Register arrays are indexed by the step number, so every step must be
// unrolled; nvcc's own unroller gives up on the 64-step nests (and then puts
// the row in local memory), template recursion does not.
template <int Begin, int End, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (Begin < End) {
        f(std::integral_constant<int, Begin>{});
        static_for<Begin + 1, End>(f);
    }
}

template <typename T> __device__ __forceinline__ T tiny_normal();
template <> __device__ __forceinline__ double tiny_normal<double>() { return DBL_MIN; }
template <> __device__ __forceinline__ float tiny_normal<float>() { return FLT_MIN; }

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Barrier over the threads that share one matrix.
template <int NW>
__device__ __forceinline__ void mat_sync() {
    if (NW == 1) __syncwarp(); else __syncthreads();
}

// Pivot key: larger |x| wins, ties -> lower position. NaN magnitudes rank
// below every number (they are chosen only when nothing else is left), and
// rows that are no longer candidates carry key -1.
template <typename T>
__device__ __forceinline__ bool key_beats(T v2, int p2, T v, int p) {
    return (v2 > v) || (v2 == v && p2 < p);
}

// Shared memory one matrix needs.
template <typename T, int NC, int NW>
struct SmallLuShared {
    T     row[2][NC];      // pivot row broadcast (double-buffered)
    T     rhs[2][4];       // solve broadcast: one value per RHS column in a chunk of 4
    T     red_v[2][NW];    // cross-warp argmax (only NW > 1)
    int   red_p[2][NW];
    int   red_s[2][NW];
    int   perm[32 * NW];   // scratch for applying ipiv in getrs
};

// Factor the rows held in `a`. tid: thread index within the matrix.
// On return: `pos` = final row position of this thread's row, the thread with
// tid == k (k < kmax) holds ipiv(k) in `my_ipiv`, `info` is LAPACK's info.
template <typename T, int NC, int NW>
__device__ __forceinline__ void small_lu_factor(T (&a)[NC], int m, int n, int tid, int& pos,
                                                int& my_ipiv, int& info,
                                                SmallLuShared<T, NC, NW>& sh) {
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int kmax = min(m, n);
    pos = (tid < m) ? tid : INT_MAX / 2;
    info = 0;
    my_ipiv = 0;
    static_for<0, NC>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        if (k >= kmax) return;
        constexpr int buf = k & 1;
        // ---- pivot search over rows still unchosen (pos >= k) ----
        T v = (pos >= k && tid < m) ? fabs(a[k]) : T(-1);
        if (v != v) v = T(-0.5);
        int p = (pos >= k && tid < m) ? pos : INT_MAX;
        int s = tid;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            T v2 = __shfl_xor_sync(kFullMask, v, off);
            int p2 = __shfl_xor_sync(kFullMask, p, off);
            int s2 = __shfl_xor_sync(kFullMask, s, off);
            if (key_beats(v2, p2, v, p)) { v = v2; p = p2; s = s2; }
        }
        if (NW > 1) {
            if (lane == 0) { sh.red_v[buf][warp] = v; sh.red_p[buf][warp] = p; sh.red_s[buf][warp] = s; }
            __syncthreads();
            v = sh.red_v[buf][0]; p = sh.red_p[buf][0]; s = sh.red_s[buf][0];
#pragma unroll
            for (int w = 1; w < NW; ++w) {
                T v2 = sh.red_v[buf][w];
                int p2 = sh.red_p[buf][w];
                if (key_beats(v2, p2, v, p)) { v = v2; p = p2; s = sh.red_s[buf][w]; }
            }
        }
        // ---- the pivot row publishes columns k..n-1 ----
        if (tid == s) {
#pragma unroll
            for (int j = k; j < NC; ++j) sh.row[buf][j] = a[j];
        }
        mat_sync<NW>();
        const T piv = sh.row[buf][k];
        // ---- LAPACK swap bookkeeping: ipiv(k) = current position of the pivot row ----
        if (tid == k) my_ipiv = p + 1;
        if (piv != T(0)) {
            if (pos == k) pos = p;   // row at position k moves to the pivot's old position
            if (tid == s) pos = k;
        } else if (info == 0) {
            info = k + 1;
        }
        // ---- scale column k below the pivot and apply the rank-1 update ----
        if (pos > k && tid < m) {
            if (piv != T(0)) {
                if (fabs(piv) >= tiny_normal<T>()) a[k] = a[k] * (T(1) / piv);
                else                               a[k] = a[k] / piv;
            }
            const T l = a[k];
#pragma unroll
            for (int j = k + 1; j < NC; ++j) {
                if (j < n) a[j] = fma_rn(l, -sh.row[buf][j], a[j]);
            }
        }
    });
}

// Solve with the factors held in registers. Each thread holds its LU row at
// position `pos`; b[r] holds the entry of right-hand side r that belongs at
// position `pos` of P*b. Forward substitution with unit L, then backward with
// U, in the operation order of reference BLAS dtrsm (Left, NoTrans):
//   b(i) = fma(-b(k), L(i,k), b(i))   for k ascending,
//   b(k) = b(k) / U(k,k);  b(i) = fma(-b(k), U(i,k), b(i))   for k descending.
template <typename T, int NC, int NW, int R>
__device__ __forceinline__ void small_lu_solve(const T (&a)[NC], int n, int pos, T (&b)[R],
                                               SmallLuShared<T, NC, NW>& sh) {
    static_for<0, NC>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        if (k >= n) return;
        constexpr int buf = k & 1;
        if (pos == k) {
#pragma unroll
            for (int r = 0; r < R; ++r) sh.rhs[buf][r] = b[r];
        }
        mat_sync<NW>();
        if (pos > k && pos < n) {
#pragma unroll
            for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.rhs[buf][r], a[k], b[r]);
        }
    });
    static_for<0, NC>([&](auto ic) {
        constexpr int kk = NC - 1 - decltype(ic)::value;
        if (kk >= n) return;
        // global step t = n + (n-1-kk); buffer t&1 == (kk+1)&1 keeps consecutive
        // steps (including the forward->backward hand-over) on different buffers
        constexpr int buf = (kk + 1) & 1;
        if (pos == kk) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                b[r] = b[r] / a[kk];
                sh.rhs[buf][r] = b[r];
            }
        }
        mat_sync<NW>();
        if (pos < kk) {
#pragma unroll
            for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.rhs[buf][r], a[kk], b[r]);
        }
    });
}

}  // namespace mb200
