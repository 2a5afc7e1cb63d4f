// chol.cuh -- Cholesky factorisation (potrf) and solve (potrs) device code.
//
// Thread i owns row i of the lower triangle (for uplo = Upper: column i of
// the upper triangle, i.e. the same numbers transposed). Step k:
//   every live row publishes its raw column-k entry to shared memory; after
//   ONE barrier each thread reads d = A(k,k), checks d > 0 (NaN fails, as
//   LAPACK's "AJJ.LE.ZERO.OR.DISNAN(AJJ)"), forms r = 1/sqrt(d) and applies
//   A(i,j) = fma(-A(i,k)*r, A(j,k)*r, A(i,j)) for k < j <= i,
// recomputing the scaled multiplier A(j,k)*r itself instead of waiting for
// its owner (same operands, same rounding). Every element sees the oracle's
// operations in the oracle's order, so factors are bit-identical.
//
// Replaces the reference's lpout Cholesky (magmablas/zpotf2_kernels_var.cu:80-111:
// one launch per 8 columns of the largest matrix) and its large-size path
// (src/zpotrf_vbatched.cpp:19-247: panel + trsm + herk launches, or a host
// loop over cuBLAS dsyrk on 32 streams).
#pragma once

#include "lu_sizes.h"
#include "small_lu.cuh"
#include <type_traits>

namespace mb200 {

template <typename T> __device__ __forceinline__ T sqrt_rn(T x);
template <> __device__ __forceinline__ double sqrt_rn<double>(double x) { return __dsqrt_rn(x); }
template <> __device__ __forceinline__ float sqrt_rn<float>(float x) { return __fsqrt_rn(x); }

template <typename T, int NC>
struct CholShared {
    alignas(16) T col[2][NC];   // raw column k (double-buffered)
    alignas(16) T row[2][NC];   // row broadcast for the transposed solve
    T rhs[2][8];                // one value per right-hand side of a group (R <= 8)
};

// Factor steps k0 .. k0+nsteps-1 on register columns 0..nsteps-1. `a` holds
// this thread's row (entries of columns k0..k0+NC-1); rows are live when
// k0 <= tid < n. Returns the 1-based failing step or 0.
// The steps run in chunks of CK: a chunk's code is unrolled over the registers
// from its first column on and looped over its CK steps at run time (the chunk's
// own columns picked by selects), which keeps the kernel small enough for the
// instruction cache; each element sees the same operations in the same order.
template <typename T, int NC, int NW, typename Sync = MatSync<NW>>
__device__ __forceinline__ int chol_panel_steps(T (&a)[NC], int n, int nsteps, int k0, int tid,
                                                CholShared<T, NC>& sh, const Sync& sync = Sync{}) {
    constexpr int CK = NC < 8 ? NC : 8;
    static_assert(NC % CK == 0, "chunking");
    int info = 0;
    static_for<0, NC / CK>([&](auto cc) {
        constexpr int c0 = decltype(cc)::value * CK;
        if (c0 >= nsteps || info != 0) return;
        const int kend = min(c0 + CK, nsteps);
#pragma unroll 1
        for (int k = c0; k < kend; ++k) {
            const int buf = k & 1;
            const int g = k0 + k;
            T ak = a[c0];
#pragma unroll
            for (int q = 1; q < CK; ++q) ak = (k == c0 + q) ? a[c0 + q] : ak;
            if (tid >= g && tid < n && tid < k0 + NC) sh.col[buf][tid - k0] = ak;
            sync();
            const T d = sh.col[buf][k];
            if (!(d > T(0))) {      // not positive definite (or NaN): stop, A(g,g) keeps d
                info = g + 1;
                break;
            }
            const T s = sqrt_rn(d);
            const T r = T(1) / s;
            const bool live = tid > g && tid < n;
            const T l = ak * r;
            const T nk = (tid == g) ? s : (live ? l : ak);
#pragma unroll
            for (int q = 0; q < CK; ++q)
                if (k == c0 + q) a[c0 + q] = nk;
            if (live) {
#pragma unroll
                for (int j = c0; j < c0 + CK; ++j)
                    if (j > k) a[j] = fma_rn(-l, sh.col[buf][j] * r, a[j]);
#pragma unroll
                for (int j = c0 + CK; j < NC; ++j) a[j] = fma_rn(-l, sh.col[buf][j] * r, a[j]);
            }
        }
    });
    return info;
}

// The same steps fully unrolled: the blocked factorisation's 32-column panel, whose
// code is small enough for the instruction cache and which spilled when chunked.
template <typename T, int NC, int NW, typename Sync = MatSync<NW>>
__device__ __forceinline__ int chol_panel_steps_unrolled(T (&a)[NC], int n, int nsteps, int k0, int tid,
                                                         CholShared<T, NC>& sh, const Sync& sync = Sync{}) {
    int info = 0;
    static_for<0, NC>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        if (k >= nsteps || info != 0) return;
        constexpr int buf = k & 1;
        const int g = k0 + k;
        if (tid >= g && tid < n && tid < k0 + NC) sh.col[buf][tid - k0] = a[k];
        sync();
        const T d = sh.col[buf][k];
        if (!(d > T(0))) {
            info = g + 1;
            return;
        }
        const T s = sqrt_rn(d);
        const T r = T(1) / s;
        if (tid == g) a[k] = s;
        if (tid > g && tid < n) {
            const T l = a[k] * r;
            a[k] = l;
#pragma unroll
            for (int j = k + 1; j < NC; ++j) a[j] = fma_rn(-l, sh.col[buf][j] * r, a[j]);
        }
    });
    return info;
}

// Solve L L^T x = b for register-resident rows of L (thread = row, `a` = row).
// Forward: b(k) *= 1/L(k,k); b(i) = fma(-b(k), L(i,k), b(i)) for i > k.
// Backward (column sweep of U = L^T): b(k) *= 1/L(k,k); b(i) = fma(-b(k), L(k,i), b(i)) for i < k,
// with row k of L published through shared memory. Chunked like chol_panel_steps.
// The diagonal enters as its correctly rounded reciprocal, formed by each thread for its
// own row before the sweeps, so no division sits on the step-to-step chain (an IEEE
// division is ~127 cycles of it on B200); the oracle's dpotrs is restated the same way.
template <typename T, int NC, int NW, int R, typename Sync = MatSync<NW>>
__device__ __forceinline__ void chol_solve(const T (&a)[NC], int n, int tid, T (&b)[R], CholShared<T, NC>& sh,
                                           const Sync& sync = Sync{}) {
    static_assert(R <= 8, "CholShared::rhs holds 8 right-hand sides a group");
    constexpr int CK = NC < 8 ? NC : 8;
    T dk = T(1);
#pragma unroll
    for (int j = 0; j < NC; ++j) dk = (j == tid) ? a[j] : dk;
    const T rk = T(1) / dk;   // this row's 1/L(tid,tid)
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
            const T ak = pick(k, std::integral_constant<int, c0>{});
            if (tid == k) {
#pragma unroll
                for (int r = 0; r < R; ++r) { b[r] = b[r] * rk; sh.rhs[buf][r] = b[r]; }
            }
            sync();
            if (tid > k && tid < n) {
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
        for (int k = ktop; k >= c0; --k) {
            const int buf = (k + 1) & 1;
            if (tid == k) {
#pragma unroll
                for (int r = 0; r < R; ++r) { b[r] = b[r] * rk; sh.rhs[buf][r] = b[r]; }
#pragma unroll
                for (int j = 0; j < c0; ++j) sh.row[buf][j] = a[j];
#pragma unroll
                for (int j = c0; j < c0 + CK; ++j)
                    if (j < k) sh.row[buf][j] = a[j];
            }
            sync();
            if (tid < k) {
                const T lki = sh.row[buf][tid];
#pragma unroll
                for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.rhs[buf][r], lki, b[r]);
            }
        }
    });
}

// Element (i, j) of the stored triangle: lower -> A(i, j), upper -> A(j, i).
template <typename T>
__device__ __forceinline__ T& tri(T* A, int lda, bool upper, int i, int j) {
    return upper ? A[j + (size_t)i * lda] : A[i + (size_t)j * lda];
}

// One instance of the register-resident kernels: potrf (thread = row, n <= NC) and,
// when SOLVE, potrs on its right-hand sides R at a time. n <= 0 writes info 0 only.
template <typename T, int NC, int NW, int R, bool SOLVE, typename Sync = MatSync<NW>>
__device__ __forceinline__ void chol_small_instance(int id, const LuSizes& sz, bool upper, T** dA_array,
                                                    T** dB_array, int* info_array, int tid, CholShared<T, NC>& sh,
                                                    const Sync& sync = Sync{}) {
    const int n = sz.get_n(id), lda = sz.get_lda(id);
    if (n <= 0) {
        if (tid == 0 && info_array) info_array[id] = 0;
        return;
    }
    T* A = dA_array[id];
    T a[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) a[j] = (tid < n && j <= tid) ? tri(A, lda, upper, tid, j) : T(0);
    // the first group of right-hand sides is loaded with A, so its latency hides behind
    // the factorisation (after the stores of A the compiler could not move it earlier)
    T b0[R];
    if constexpr (SOLVE) {
        const int nrhs0 = sz.get_nrhs(id), ldb0 = sz.get_ldb(id);
        const T* B0 = dB_array[id];
#pragma unroll
        for (int r = 0; r < R; ++r) b0[r] = (tid < n && r < nrhs0) ? B0[tid + (size_t)r * ldb0] : T(0);
    }
    const int info = chol_panel_steps<T, NC, NW>(a, n, n, 0, tid, sh, sync);
    if (tid < n) {
        // on failure the rows stay as the steps left them, like LAPACK's partial factor
#pragma unroll
        for (int j = 0; j < NC; ++j)
            if (j <= tid) tri(A, lda, upper, tid, j) = a[j];
    }
    if (tid == 0 && info_array) info_array[id] = info;
    if constexpr (SOLVE) {
        // MAGMA's posv solves regardless of info (src/zposv_batched.cpp:123-141)
        T* B = dB_array[id];
        const int nrhs = sz.get_nrhs(id), ldb = sz.get_ldb(id);
        for (int c0 = 0; c0 < nrhs; c0 += R) {
            T b[R];
#pragma unroll
            for (int r = 0; r < R; ++r)
                b[r] = (c0 == 0) ? b0[r] : (tid < n && c0 + r < nrhs) ? B[tid + (size_t)(c0 + r) * ldb] : T(0);
            chol_solve<T, NC, NW, R>(a, n, tid, b, sh, sync);
            if (tid < n) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (c0 + r < nrhs) B[tid + (size_t)(c0 + r) * ldb] = b[r];
            }
        }
    }
}

// One instance of potrs alone with the factor's rows in registers.
template <typename T, int NC, int NW, int R, typename Sync = MatSync<NW>>
__device__ __forceinline__ void potrs_small_instance(int id, const LuSizes& sz, bool upper, T** dA_array,
                                                     T** dB_array, int tid, CholShared<T, NC>& sh,
                                                     const Sync& sync = Sync{}) {
    const int n = sz.get_n(id), lda = sz.get_lda(id), nrhs = sz.get_nrhs(id), ldb = sz.get_ldb(id);
    if (n <= 0 || nrhs <= 0) return;
    T* A = dA_array[id];
    T* B = dB_array[id];
    T a[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) a[j] = (tid < n && j <= tid) ? tri(A, lda, upper, tid, j) : T(0);
    for (int c0 = 0; c0 < nrhs; c0 += R) {
        T b[R];
#pragma unroll
        for (int r = 0; r < R; ++r) b[r] = (tid < n && c0 + r < nrhs) ? B[tid + (size_t)(c0 + r) * ldb] : T(0);
        chol_solve<T, NC, NW, R>(a, n, tid, b, sh, sync);
        if (tid < n) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (c0 + r < nrhs) B[tid + (size_t)(c0 + r) * ldb] = b[r];
        }
    }
}

// ---------------------------------------------------------------------------
// Blocked right-looking Cholesky of one matrix per thread block (n <= NT).
// Per panel of NB columns: thread t factors row t's panel entries in registers
// (chol_panel_steps), every row publishes them to shared memory, and the
// trailing lower triangle A22 -= P P^T is computed by all threads in 4x8 tiles
// distributed evenly over the triangle (a row-per-thread update would leave
// the last rows with most of the work). Each element still receives
// fma(-L(i,r), L(j,r), a) for r ascending, the unblocked order.
template <typename T, int NB, int NT, int CW>
struct BlockedCholShared {
    CholShared<T, NB> p;
    T P[NT][NB + 1];     // panel entries of every row
};

// One FP64 tensor-core step D = A B + D on an 8x8 tile (mma.sync m8n8k4: lane l holds
// A(l/4, l%4), B(l%4, l/4) and D(l/4, 2(l%4) .. +1)); each element of D receives its four
// products as fma's in ascending k, rounded after each (the unblocked order).
__device__ __forceinline__ void chol_dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// Trailing update of one panel on the FP64 tensor cores: A22 -= P P^T on the lower
// triangle from row/column m0 on, in jobs of 32 rows x 8 columns per warp (four 8x8
// accumulator tiles, so four independent MMA chains). The multipliers come from the
// panel rows in shared memory (A fragment negated: (-l_i) l_j + a is the fma of the
// CUDA-core update), steps past the panel's nbp are zero, and each element receives its
// nbp updates in ascending order, exactly as in the CUDA-core update. With PREFETCH the
// next job's entries are loaded before the current job's products (16 more registers a
// thread; the persistent queue kernel, whose every path shares one 128-register budget,
// spills with it and loads each job's entries in turn instead).
template <int NB, int NT, int CW, bool PREFETCH, typename Team>
__device__ __forceinline__ void chol_update_dmma(double* __restrict__ A, int n, int lda, bool upper, int m0,
                                                 int nbp, const BlockedCholShared<double, NB, NT, CW>& sh,
                                                 const Team& team) {
    constexpr int NW = NT / 32;
    const int tid = team.tid(), lane = tid & 31, warp = tid >> 5;
    const int q = lane & 3, r8 = lane >> 2;
    const int T8 = (n - m0 + 7) / 8;   // 8-column tiles of the trailing triangle
    // element (i, j) of the stored triangle at A + i * si + j * sj (lower: A(i, j); upper: A(j, i))
    const size_t si = upper ? (size_t)lda : 1, sj = upper ? 1 : (size_t)lda;
    auto load_c = [&](int bj, int rb, double (&c)[4][2]) {
        const int j0 = m0 + 8 * bj, ib = j0 + 32 * rb;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const int i = ib + 8 * g + r8;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = j0 + 2 * q + h;
                c[g][h] = (i < n && j <= i) ? A[i * si + j * sj] : 0.0;
            }
        }
    };
    int job = 0;
    double cn[4][2];
    // the warp's jobs in order: (bj, rb) with rb < ceil((T8 - bj) / 4), every NW-th job
    auto next_job = [&](int& bj, int& rb) {
        while (bj < T8) {
            const int nrb = (T8 - bj + 3) / 4;
            while (rb < nrb) {
                if (job++ % NW == warp) return true;
                ++rb;
            }
            ++bj;
            rb = 0;
        }
        return false;
    };
    int bj = 0, rb = 0;
    bool have = next_job(bj, rb);
    if (PREFETCH && have) load_c(bj, rb, cn);
    while (have) {
        double cc[4][2];
        if constexpr (PREFETCH) {
#pragma unroll
            for (int g = 0; g < 4; ++g) { cc[g][0] = cn[g][0]; cc[g][1] = cn[g][1]; }
        } else {
            load_c(bj, rb, cc);
        }
        const int cbj = bj, crb = rb;
        ++rb;
        have = next_job(bj, rb);
        if (PREFETCH && have) load_c(bj, rb, cn);   // in flight while the current job computes
        const int j0 = m0 + 8 * cbj, ib = j0 + 32 * crb;
#pragma unroll
        for (int s4 = 0; s4 < NB / 4; ++s4) {
            const int kk = 4 * s4 + q;
            const bool kv = kk < nbp;
            const double b = kv ? sh.P[min(j0 + r8, NT - 1)][kk] : 0.0;
            double af[4];
#pragma unroll
            for (int g = 0; g < 4; ++g) af[g] = kv ? -sh.P[min(ib + 8 * g + r8, NT - 1)][kk] : 0.0;
#pragma unroll
            for (int g = 0; g < 4; ++g) chol_dmma(cc[g][0], cc[g][1], af[g], b);
        }
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const int i = ib + 8 * g + r8;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = j0 + 2 * q + h;
                if (i < n && j <= i) A[i * si + j * sj] = cc[g][h];
            }
        }
    }
}

template <typename T, int NB, int NT, int CW, int CB, typename Team = BlockTeam, bool DMMA = false,
          bool PREFETCH = true>
__device__ int blocked_potrf(T* __restrict__ A, int n, int lda, bool upper, BlockedCholShared<T, NB, NT, CW>& sh,
                             const Team& team = Team{}) {
    constexpr int NW = NT / 32;
    // tile rows x columns; 2 rows when the block size leaves 64 registers a thread (FP64)
    constexpr int TR = (NT >= 1024 && sizeof(T) == 8) ? 2 : 4, TC = 8, G = 8 / TR;
    const int tid = team.tid();
    auto sync = [&] { team.sync(); };
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int nbp = min(NB, n - k0);
        const bool live = (tid >= k0 && tid < n);
        T a[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c)
            a[c] = (live && c < nbp && k0 + c <= tid) ? tri(A, lda, upper, tid, k0 + c) : T(0);
        const int info = chol_panel_steps_unrolled<T, NB, NW>(a, n, nbp, k0, tid, sh.p, sync);
        if (live) {
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if (c < nbp && k0 + c <= tid) tri(A, lda, upper, tid, k0 + c) = a[c];
#pragma unroll
            for (int c = 0; c < NB; ++c) sh.P[tid][c] = a[c];
        }
        if (info) return info;
        team.sync();
        // trailing lower triangle: rows/columns m0..n-1, square 8x8 blocks (bj <= bi),
        // each split into G work items of TR rows
        const int m0 = k0 + nbp;
        if constexpr (DMMA && std::is_same<T, double>::value) {
            chol_update_dmma<NB, NT, CW, PREFETCH>(A, n, lda, upper, m0, nbp, sh, team);
            team.sync();   // trailing entries visible before the next panel loads them
            continue;
        }
        const int T8 = (n - m0 + 7) / 8;
        const int items = G * T8 * (T8 + 1) / 2;
        for (int w = tid; w < items; w += NT) {
            const int blk = w / G, h = w % G;
            int bi = (int)((sqrtf(8.0f * blk + 1.0f) - 1.0f) * 0.5f);
            while ((bi + 1) * (bi + 2) / 2 <= blk) ++bi;
            while (bi * (bi + 1) / 2 > blk) --bi;
            const int bj = blk - bi * (bi + 1) / 2;
            const int i0 = m0 + 8 * bi + TR * h, j0 = m0 + 8 * bj;
            T acc[TR][TC];
#pragma unroll
            for (int ii = 0; ii < TR; ++ii)
#pragma unroll
                for (int jj = 0; jj < TC; ++jj) {
                    const int i = i0 + ii, j = j0 + jj;
                    acc[ii][jj] = (i < n && j <= i) ? tri(A, lda, upper, i, j) : T(0);
                }
            for (int r = 0; r < nbp; ++r) {
                T li[TR], lj[TC];
#pragma unroll
                for (int ii = 0; ii < TR; ++ii) li[ii] = sh.P[min(i0 + ii, NT - 1)][r];
#pragma unroll
                for (int jj = 0; jj < TC; ++jj) lj[jj] = sh.P[min(j0 + jj, NT - 1)][r];
#pragma unroll
                for (int ii = 0; ii < TR; ++ii)
#pragma unroll
                    for (int jj = 0; jj < TC; ++jj) acc[ii][jj] = fma_rn(-li[ii], lj[jj], acc[ii][jj]);
            }
#pragma unroll
            for (int ii = 0; ii < TR; ++ii)
#pragma unroll
                for (int jj = 0; jj < TC; ++jj) {
                    const int i = i0 + ii, j = j0 + jj;
                    if (i < n && j <= i) tri(A, lda, upper, i, j) = acc[ii][jj];
                }
        }
        team.sync();   // trailing entries visible before the next panel loads them
    }
    return 0;
}

// Blocked L L^T x = b for one matrix per thread block (n <= NT), R RHS at a time.
template <typename T, int NT, int R>
struct BlockedCholRsShared {
    T sb[32][R];
    T D[32][33];
    T rD[32];   // 1 / D(i,i) of the current diagonal block
};

// The warp that owns diagonal block [j0, j0+cnt) loads it into shared memory (rows past
// cnt: zero) with its reciprocals: the loads go out unconditionally, clamped inside the
// matrix, 8 at a time, so they overlap instead of completing one by one.
template <typename T, int NT, int R, typename F>
__device__ __forceinline__ void load_diag_block(BlockedCholRsShared<T, NT, R>& sh, int cnt, int lane, F&& Lb) {
    const int li = min(lane, cnt - 1);
#pragma unroll
    for (int c0 = 0; c0 < 32; c0 += 8) {
        T v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = Lb(li, min(c0 + c, cnt - 1));
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c0 + c <= lane && lane < cnt) sh.D[lane][c0 + c] = v[c];
    }
    if (lane < cnt) sh.rD[lane] = T(1) / Lb(lane, lane);
    __syncwarp();
}

template <typename T, int NT, int R, typename Team = BlockTeam>
__device__ void blocked_potrs(const T* __restrict__ A, int n, int lda, bool upper, T* __restrict__ B, int nrhs,
                              int ldb, BlockedCholRsShared<T, NT, R>& sh, const Team& team = Team{}) {
    const int t = team.tid(), lane = t & 31;
    const int nblk = (n + 31) / 32;
    auto L = [&](int i, int j) -> T { return upper ? A[j + (size_t)i * lda] : A[i + (size_t)j * lda]; };
    for (int c0 = 0; c0 < nrhs; c0 += R) {
        T b[R];
#pragma unroll
        for (int r = 0; r < R; ++r) b[r] = (t < n && c0 + r < nrhs) ? B[t + (size_t)(c0 + r) * ldb] : T(0);
        // forward: L y = b, blocks ascending
        for (int J = 0; J < nblk; ++J) {
            const int j0 = J * 32, j1 = min(n, j0 + 32), cnt = j1 - j0;
            team.sync();
            if ((t >> 5) == J) {
                load_diag_block(sh, cnt, lane, [&](int i, int j) { return L(j0 + i, j0 + j); });
                // steps unrolled over the block (no loop or branch overhead on the chain)
                static_for<0, 32>([&](auto kc) {
                    constexpr int k = decltype(kc)::value;
                    if (k >= cnt) return;
                    if (lane == k) {
#pragma unroll
                        for (int r = 0; r < R; ++r) { b[r] = b[r] * sh.rD[k]; sh.sb[k][r] = b[r]; }
                    }
                    __syncwarp();
                    if (lane > k && lane < cnt) {
                        const T l = sh.D[lane][k];
#pragma unroll
                        for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.sb[k][r], l, b[r]);
                    }
                });
            }
            team.sync();
            if (t >= j1 && t < n)
                block_update<T, R, false>(b, sh.sb, cnt, [&](int q) { return L(t, j0 + q); });
        }
        // backward: L^T x = y, blocks descending (column sweep of U = L^T)
        for (int J = nblk - 1; J >= 0; --J) {
            const int j0 = J * 32, j1 = min(n, j0 + 32), cnt = j1 - j0;
            team.sync();
            if ((t >> 5) == J) {
                load_diag_block(sh, cnt, lane, [&](int i, int j) { return L(j0 + i, j0 + j); });
                static_for<0, 32>([&](auto kc) {
                    constexpr int k = 31 - decltype(kc)::value;
                    if (k >= cnt) return;
                    if (lane == k) {
#pragma unroll
                        for (int r = 0; r < R; ++r) { b[r] = b[r] * sh.rD[k]; sh.sb[k][r] = b[r]; }
                    }
                    __syncwarp();
                    if (lane < k) {
                        const T u = sh.D[k][lane];   // U(t, k) = L(k, t)
#pragma unroll
                        for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.sb[k][r], u, b[r]);
                    }
                });
            }
            team.sync();
            if (t < j0)
                block_update<T, R, true>(b, sh.sb, cnt, [&](int q) { return L(j0 + q, t); });
        }
        if (t < n) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (c0 + r < nrhs) B[t + (size_t)(c0 + r) * ldb] = b[r];
        }
        team.sync();
    }
}

}  // namespace mb200
