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

// Asks L2 to fetch [p, p + bytes) ahead of use, without waiting and without
// registers: a bulk prefetch through the copy engine when p is 16-byte aligned
// (the size rounded down to whole 16-byte units), else one line at a time.
// Every byte of the range must lie inside the caller's allocation.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    if ((a & 15) == 0) {
        const unsigned sz = bytes & ~15u;
        if (sz) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(sz) : "memory");
    } else {
        for (unsigned off = 0; off < bytes; off += 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char*>(p) + off));
    }
}

// Barrier over the threads that share one matrix.
template <int NW>
__device__ __forceinline__ void mat_sync() {
    if (NW == 1) __syncwarp(); else __syncthreads();
}

// The threads that share one matrix as a barrier functor: the whole block or one
// warp (MatSync), or a team of warps inside a larger block (BarSync: a named
// barrier of `count` threads, which orders their shared-memory accesses as
// __syncthreads does for the block).
template <int NW>
struct MatSync {
    __device__ __forceinline__ void operator()() const { mat_sync<NW>(); }
};
struct BarSync {
    int id, count;
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
    }
};

// A matrix's threads for the one-matrix-per-team kernels: rank within the team and
// the team's barrier. BlockTeam is the whole thread block; WarpRangeTeam is the
// warps [first, first + count / 32) of a larger block on named barrier `id`.
struct BlockTeam {
    __device__ __forceinline__ int tid() const { return threadIdx.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct WarpRangeTeam {
    int first_thread, id, count;
    __device__ __forceinline__ int tid() const { return threadIdx.x - first_thread; }
    __device__ __forceinline__ void sync() const { BarSync{id, count}(); }
};

// Pivot key: |x| as an ordered unsigned integer (the bit pattern of a
// non-negative IEEE number is monotonic in its value), split into two 32-bit
// halves for the warp REDUX instructions. Order: rows that are not candidates
// (key 0, position INT_MAX) < NaN (key 0) < 0 (key 1) < ... < +inf. Among
// equal keys the lowest row position wins, which is IDAMAX's first-maximum rule.
struct PivotKey { unsigned hi, lo; };

__device__ __forceinline__ PivotKey pivot_key(double x, bool cand) {
    const double v = fabs(x);
    unsigned long long b = (cand && v == v) ? (unsigned long long)__double_as_longlong(v) + 1ull : 0ull;
    return {unsigned(b >> 32), unsigned(b)};
}
__device__ __forceinline__ PivotKey pivot_key(float x, bool cand) {
    const float v = fabsf(x);
    return {(cand && v == v) ? unsigned(__float_as_uint(v)) + 1u : 0u, 0u};
}

__device__ __forceinline__ bool key_beats(PivotKey k2, int p2, PivotKey k, int p) {
    return (k2.hi > k.hi) || (k2.hi == k.hi && (k2.lo > k.lo || (k2.lo == k.lo && p2 < p)));
}

// Warp-wide argmax: on return every lane holds the winning key and position;
// the result is the lane that holds the winner.
__device__ __forceinline__ int warp_argmax(PivotKey& key, int& p, int lane) {
    (void)lane;
    const unsigned mhi = __reduce_max_sync(kFullMask, key.hi);
    const unsigned mlo = __reduce_max_sync(kFullMask, key.hi == mhi ? key.lo : 0u);
    const bool top = (key.hi == mhi && key.lo == mlo);
    const int pmin = __reduce_min_sync(kFullMask, top ? p : INT_MAX);
    const unsigned who = __ballot_sync(kFullMask, top && p == pmin);
    key.hi = mhi;
    key.lo = mlo;
    p = pmin;
    return __ffs(who) - 1;
}

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };
template <typename T> __device__ __forceinline__ typename Vec2<T>::type make_vec2(T x, T y);
template <> __device__ __forceinline__ double2 make_vec2<double>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 make_vec2<float>(float x, float y) { return make_float2(x, y); }

// b[r] -= sb[kk][r] * f(kk) for the cnt (<= 32) entries of one 32-row block, as
// single fma's in ascending kk (or descending when DESC). The factor entries
// are loaded in groups of 16 with clamped, always-valid indices, so a group's
// loads are issued together instead of one load -> fma dependency per entry.
template <typename T, int R, bool DESC, typename F>
__device__ __forceinline__ void block_update(T (&b)[R], const T (&sb)[32][R], int cnt, F&& f) {
    constexpr int G = 16;
#pragma unroll
    for (int g = 0; g < 32; g += G) {
        const int base = DESC ? 32 - G - g : g;
        T v[G];
#pragma unroll
        for (int q = 0; q < G; ++q) v[q] = f(min(base + q, cnt - 1));
#pragma unroll
        for (int qq = 0; qq < G; ++qq) {
            const int q = DESC ? G - 1 - qq : qq;
            if (base + q < cnt) {
#pragma unroll
                for (int r = 0; r < R; ++r) b[r] = fma_rn(-sb[base + q][r], v[q], b[r]);
            }
        }
    }
}

// Shared memory one matrix needs.
template <typename T, int NC, int NW>
struct SmallLuShared {
    static_assert(NC % 2 == 0, "the pivot row is broadcast in pairs");
    alignas(16) T row[2][NC];   // pivot row broadcast (double-buffered)
    T        rhs[2][4];         // solve broadcast: one value per RHS column in a chunk of 4
    unsigned red_hi[2][NW];     // cross-warp argmax (only NW > 1)
    unsigned red_lo[2][NW];
    int      red_p[2][NW];
    int      red_s[2][NW];
};

// Eliminate register columns 0..nsteps-1 of the rows held in `a` (updating
// columns up to ncols-1), as global elimination steps g = k0 .. k0+nsteps-1
// (k0 = 0 for a whole small matrix; the panel offset in the blocked
// factorisation). tid: thread index within the
// matrix; `pos` must hold the thread's current row position on entry (tid for
// live rows, anything < k0 for finished rows, a huge value for tid >= m).
// On return `pos` is the row's new position, the thread with tid == g holds
// ipiv(g) (1-based) in `my_ipiv`, and `info` is g+1 of the first zero pivot.
// With nopiv the row at position g is step g's pivot (getrf_nopiv): no search,
// rows never change position.
template <typename T, int NC, int NW, typename Sync = MatSync<NW>>
__device__ __forceinline__ void lu_panel_steps(T (&a)[NC], int m, int nsteps, int ncols, int k0, int tid, int& pos,
                                               int& my_ipiv, int& info,
                                               SmallLuShared<T, NC, NW>& sh, bool nopiv = false,
                                               const Sync& sync = Sync{}) {
    (void)ncols;   // columns >= ncols hold zeros in every row, so their updates are no-ops
    const int lane = tid & 31;
    const int warp = tid >> 5;
    using V2 = typename Vec2<T>::type;
    static_for<0, NC>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        if (k >= nsteps) return;
        constexpr int buf = k & 1;
        const int g = k0 + k;
        // ---- pivot search over rows still unchosen (pos >= g) ----
        int p = g, s = g;
        if (!nopiv) {
        const bool cand = (pos >= g && tid < m);
        PivotKey key = pivot_key(a[k], cand);
        p = cand ? pos : INT_MAX;
        s = warp_argmax(key, p, lane) + warp * 32;
        if (NW > 1) {
            if (lane == 0) { sh.red_hi[buf][warp] = key.hi; sh.red_lo[buf][warp] = key.lo; sh.red_p[buf][warp] = p; sh.red_s[buf][warp] = s; }
            sync();
            // every warp reduces the NW warp winners lane-parallel (lane w = warp w's winner)
            const bool v = lane < NW;
            key = PivotKey{v ? sh.red_hi[buf][lane] : 0u, v ? sh.red_lo[buf][lane] : 0u};
            p = v ? sh.red_p[buf][lane] : INT_MAX;
            s = sh.red_s[buf][warp_argmax(key, p, lane)];
        }
        }
        // ---- the pivot row publishes columns k..NC-1 (aligned pairs) ----
        constexpr int jw = k & ~1;
        if (tid == s) {
            V2* row2 = reinterpret_cast<V2*>(&sh.row[buf][0]);
#pragma unroll
            for (int j = jw; j < NC; j += 2) row2[j / 2] = make_vec2<T>(a[j], a[j + 1]);
        }
        sync();
        const T piv = sh.row[buf][k];
        // ---- LAPACK swap bookkeeping: ipiv(g) = current position of the pivot row ----
        if (tid == g) my_ipiv = p + 1;
        if (piv != T(0)) {
            if (pos == g) pos = p;   // row at position g moves to the pivot's old position
            if (tid == s) pos = g;
        } else if (info == 0) {
            info = g + 1;
        }
        // ---- scale column k below the pivot and apply the rank-1 update ----
        if (pos > g && tid < m) {
            if (piv != T(0)) {
                if (fabs(piv) >= tiny_normal<T>()) a[k] = a[k] * (T(1) / piv);
                else                               a[k] = a[k] / piv;
            }
            const T l = a[k];
            const V2* row2 = reinterpret_cast<const V2*>(&sh.row[buf][0]);
#pragma unroll
            for (int j = (k + 1) & ~1; j < NC; j += 2) {
                const V2 u = row2[j / 2];
                if (j > k) a[j] = fma_rn(l, -u.x, a[j]);
                a[j + 1] = fma_rn(l, -u.y, a[j + 1]);
            }
        }
    });
}

// The steps of lu_panel_steps for wide rows (NC > 32), in chunks of CK = 8: the code
// of a chunk is unrolled over the registers from the chunk's first column on and
// looped over its 8 steps at run time (the step's own column picked by selects), so
// the kernel fits the instruction cache (the fully unrolled 64-column form thrashed
// it). Every element receives the same operations in the same order.
template <typename T, int NC, int NW>
__device__ __forceinline__ void lu_panel_steps_chunked(T (&a)[NC], int m, int nsteps, int tid, int& pos,
                                                       int& my_ipiv, int& info, SmallLuShared<T, NC, NW>& sh,
                                                       bool nopiv) {
    constexpr int CK = 8;
    static_assert(NC % CK == 0, "chunking");
    const int lane = tid & 31;
    const int warp = tid >> 5;
    using V2 = typename Vec2<T>::type;
    static_for<0, NC / CK>([&](auto cc) {
        constexpr int c0 = decltype(cc)::value * CK;
        if (c0 >= nsteps) return;
        const int kend = min(c0 + CK, nsteps);
#pragma unroll 1
        for (int k = c0; k < kend; ++k) {
            const int buf = k & 1;
            const int g = k;
            T ak = a[c0];
#pragma unroll
            for (int q = 1; q < CK; ++q) ak = (k == c0 + q) ? a[c0 + q] : ak;
            int p = g, s = g;
            if (!nopiv) {
                const bool cand = (pos >= g && tid < m);
                PivotKey key = pivot_key(ak, cand);
                p = cand ? pos : INT_MAX;
                s = warp_argmax(key, p, lane) + warp * 32;
                if (NW > 1) {
                    if (lane == 0) {
                        sh.red_hi[buf][warp] = key.hi; sh.red_lo[buf][warp] = key.lo;
                        sh.red_p[buf][warp] = p; sh.red_s[buf][warp] = s;
                    }
                    __syncthreads();
                    const bool v = lane < NW;
                    key = PivotKey{v ? sh.red_hi[buf][lane] : 0u, v ? sh.red_lo[buf][lane] : 0u};
                    p = v ? sh.red_p[buf][lane] : INT_MAX;
                    s = sh.red_s[buf][warp_argmax(key, p, lane)];
                }
            }
            // the pivot row publishes columns c0..NC-1 (aligned pairs; consumers read k.. only)
            if (tid == s) {
                V2* row2 = reinterpret_cast<V2*>(&sh.row[buf][0]);
#pragma unroll
                for (int j = c0; j < NC; j += 2) row2[j / 2] = make_vec2<T>(a[j], a[j + 1]);
            }
            mat_sync<NW>();
            const T piv = sh.row[buf][k];
            if (tid == g) my_ipiv = p + 1;
            if (piv != T(0)) {
                if (pos == g) pos = p;
                if (tid == s) pos = g;
            } else if (info == 0) {
                info = g + 1;
            }
            if (pos > g && tid < m) {
                if (piv != T(0)) {
                    if (fabs(piv) >= tiny_normal<T>()) ak = ak * (T(1) / piv);
                    else                               ak = ak / piv;
                }
#pragma unroll
                for (int q = 0; q < CK; ++q)
                    if (k == c0 + q) a[c0 + q] = ak;
                const T l = ak;
                const V2* row2 = reinterpret_cast<const V2*>(&sh.row[buf][0]);
#pragma unroll
                for (int j = c0; j < NC; j += 2) {
                    const V2 u = row2[j / 2];
                    if (j > k) a[j] = fma_rn(l, -u.x, a[j]);
                    if (j + 1 > k) a[j + 1] = fma_rn(l, -u.y, a[j + 1]);
                }
            }
        }
    });
}

// Whole small matrix (m rows, n <= NC columns): steps 0 .. min(m,n)-1.
template <typename T, int NC, int NW>
__device__ __forceinline__ void small_lu_factor(T (&a)[NC], int m, int n, int tid, int& pos,
                                                int& my_ipiv, int& info,
                                                SmallLuShared<T, NC, NW>& sh, bool nopiv = false) {
    pos = (tid < m) ? tid : INT_MAX / 2;
    info = 0;
    my_ipiv = 0;
    if constexpr (NC > 32) lu_panel_steps_chunked<T, NC, NW>(a, m, min(m, n), tid, pos, my_ipiv, info, sh, nopiv);
    else lu_panel_steps<T, NC, NW>(a, m, min(m, n), n, 0, tid, pos, my_ipiv, info, sh, nopiv);
}

// small_lu_solve for wide rows (NC > 32), chunked like lu_panel_steps_chunked.
template <typename T, int NC, int NW, int R>
__device__ __forceinline__ void small_lu_solve_chunked(const T (&a)[NC], int n, int pos, T (&b)[R],
                                                       SmallLuShared<T, NC, NW>& sh) {
    constexpr int CK = 8;
    auto pick = [&](int k, auto c0c) {
        constexpr int c0 = decltype(c0c)::value;
        T ak = a[c0];
#pragma unroll
        for (int q = 1; q < CK; ++q) ak = (k == c0 + q) ? a[c0 + q] : ak;
        return ak;
    };
    static_for<0, NC / CK>([&](auto cc) {
        constexpr int c0 = decltype(cc)::value * CK;
        if (c0 >= n) return;
        const int kend = min(c0 + CK, n);
#pragma unroll 1
        for (int k = c0; k < kend; ++k) {
            const int buf = k & 1;
            if (pos == k) {
#pragma unroll
                for (int r = 0; r < R; ++r) sh.rhs[buf][r] = b[r];
            }
            mat_sync<NW>();
            if (pos > k && pos < n) {
                const T ak = pick(k, std::integral_constant<int, c0>{});
#pragma unroll
                for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.rhs[buf][r], ak, b[r]);
            }
        }
    });
    static_for<0, NC / CK>([&](auto ic) {
        constexpr int c0 = (NC / CK - 1 - decltype(ic)::value) * CK;
        if (c0 >= n) return;
        const int ktop = min(c0 + CK, n) - 1;
#pragma unroll 1
        for (int kk = ktop; kk >= c0; --kk) {
            const int buf = (kk + 1) & 1;
            if (pos == kk) {
                const T ak = pick(kk, std::integral_constant<int, c0>{});
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    b[r] = b[r] / ak;
                    sh.rhs[buf][r] = b[r];
                }
            }
            mat_sync<NW>();
            if (pos < kk) {
                const T ak = pick(kk, std::integral_constant<int, c0>{});
#pragma unroll
                for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.rhs[buf][r], ak, b[r]);
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
    static_assert(R <= 4, "SmallLuShared::rhs holds 4 right-hand sides a group");
    if constexpr (NC > 32) {
        small_lu_solve_chunked<T, NC, NW, R>(a, n, pos, b, sh);
        return;
    }
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
