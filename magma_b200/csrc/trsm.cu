// trsm.cu -- variable-size batched triangular solve and triangular multiply
// (magmablas_{d,s}trsm_vbatched*, magmablas/ztrsm_vbatched.cpp:21-215;
//  magmablas_{d,s}trmm_vbatched*, magmablas/ztrmm_vbatched.cpp:21-90).
//
// Every call is turned into a LEFT problem on an nr x nr triangle T and an nr x nc
// right-hand side X: side = Left gives T = op(A), X = B (nr = m, nc = n); side = Right
// gives T = op(A)^T, X = B^T (nr = n, nc = m), read and written through a transposed
// view, never copied. Rows are renumbered q = i or q = nr-1-i so that
//   trsm: T is lower in q (solve order = ascending q),
//   trmm: T is upper in q (row q uses rows q' >= q, so ascending q is safe in place).
// One block of 64 threads per (instance, 32-column panel of X) walks 32-row tiles in
// ascending q. A tile's accumulation runs as a 32x32 register-tiled product over
// 32-row chunks staged in shared memory (4x4 outputs a thread); trsm then solves the
// tile's diagonal block with one warp (lane = column, the 32 partial sums in
// registers) and writes the tile before the next one reads it.
//
// Order of operations (the oracle restates it): trsm, per element,
//   s = alpha * b;  s = fma(-T(q,q'), x(q'), s) for q' < q ascending;  x = s * (1 / T(q,q))
// (unit: the reciprocal is 1); trmm, per element,
//   s = 0;  s = fma(T(q,q'), b(q'), s) for q' >= q ascending;  x = alpha * s.
// The reference divides by the diagonal inside its own GPU kernels' inverted diagonal
// blocks; both agree with BLAS dtrsm/dtrmm to rounding. alpha = 0 sets X to zero
// (A not read), as BLAS does.
#include "internal.h"
#include "vbatched.h"
#include <algorithm>

namespace mb200 {

template <typename T>
struct TriArgs {
    const T* const* A;
    T** B;
    const int *m, *n, *lda, *ldb;   // per-instance sizes (variable size), or null:
    int m0, n0, lda0, ldb0;         // the sizes shared by every instance (fixed size)
    T alpha;
    bool left, unit;
};

constexpr int kTriTile = 32, kTriThreads = 64;

// FLIP: q = nr-1-i.  TT: T(i,k) = A(k,i).  BT: X(i,c) = B(c,i).  SOLVE: trsm (else trmm).
template <typename T, bool SOLVE, bool FLIP, bool TT, bool BT>
__global__ void __launch_bounds__(kTriThreads)
tri_panel_kernel(TriArgs<T> g, int panels, int batch) {
    constexpr int TS = kTriTile;
    __shared__ T sT[TS][TS + 1];   // [k][row] chunk of T
    __shared__ T sX[TS][TS + 1];   // [k][col] chunk of X
    __shared__ T sS[TS][TS + 1];   // [row][col] the tile's sums / results
    __shared__ T sD[TS][TS + 1];   // [row][k] diagonal block of T (trsm)
    __shared__ T rcp[TS];
    const int id = blockIdx.x / panels, panel = blockIdx.x - id * panels;
    if (id >= batch) return;
    const int m = g.m ? g.m[id] : g.m0, n = g.n ? g.n[id] : g.n0;
    const int nr = g.left ? m : n, nc = g.left ? n : m;
    const int c0 = panel * TS;
    if (nr <= 0 || c0 >= nc) return;
    const int C = min(TS, nc - c0);
    const int lda = g.lda ? g.lda[id] : g.lda0, ldb = g.ldb ? g.ldb[id] : g.ldb0;
    const T* A = g.A[id];
    T* B = g.B[id];
    const int tid = threadIdx.x, tx = tid % 8, ty = tid / 8;
    auto row_of = [&](int q) { return FLIP ? nr - 1 - q : q; };
    auto xaddr = [&](int q, int c) -> T* {
        const int i = row_of(q);
        return BT ? B + c + (size_t)i * ldb : B + i + (size_t)c * ldb;
    };
    auto tval = [&](int q, int qk) -> T {
        const int i = row_of(q), k = row_of(qk);
        return TT ? A[k + (size_t)i * lda] : A[i + (size_t)k * lda];
    };
    // element e of a 32x32 chunk -> (fast, slow) so that consecutive threads touch
    // consecutive addresses of the global operand
    if (g.alpha == T(0)) {
        for (int e = tid; e < nr * C; e += kTriThreads) {
            const int q = BT ? e / C : e % nr, c = BT ? e % C : e / nr;
            *xaddr(q, c0 + c) = T(0);
        }
        return;
    }
    const int ntiles = (nr + TS - 1) / TS;
    for (int tq = 0; tq < ntiles; ++tq) {
        const int q0 = tq * TS, R = min(TS, nr - q0);
        T acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int r = tx + 8 * a, c = ty * 4 + b;
                acc[a][b] = (SOLVE && r < R && c < C) ? g.alpha * *xaddr(q0 + r, c0 + c) : T(0);
            }
        if (SOLVE) {
            // the diagonal block (rows past nr: identity) and its reciprocals
            for (int e = tid; e < TS * TS; e += kTriThreads) {
                const int r = TT ? e / TS : e % TS, k = TT ? e % TS : e / TS;
                T v = T(0);
                if (r == k) v = (r < R && !g.unit) ? tval(q0 + r, q0 + k) : T(1);
                else if (k < r && r < R) v = tval(q0 + r, q0 + k);
                sD[r][k] = v;
            }
        }
        // chunks: trsm the tiles before this one, trmm this tile and the ones after it
        const int kc_begin = SOLVE ? 0 : tq, kc_end = SOLVE ? tq : ntiles;
        // trmm: the next chunk is fetched into registers while the current one is used;
        // trsm loads each chunk straight into shared memory (the registers a prefetch
        // needs cost it occupancy around its serial diagonal solves: measured slower)
        constexpr bool PREFETCH = !SOLVE;
        constexpr int EPT = TS * TS / kTriThreads;
        constexpr int EPR = PREFETCH ? EPT : 1;
        T rt[EPR], rx[EPR];
        // element u of this thread's share of chunk kc: its T and X values
        auto chunk_vals = [&](int kc, int u, T& tv, T& xv) {
            const int k0 = kc * TS, K = min(TS, nr - k0);
            const int e = tid + u * kTriThreads;
            const int r = TT ? e / TS : e % TS, kk = TT ? e % TS : e / TS;
            T v = T(0);
            if (r < R && kk < K) {
                const int q = q0 + r, qk = k0 + kk;
                if (SOLVE) v = tval(q, qk);                          // qk < q0 <= q
                else if (qk > q) v = tval(q, qk);
                else if (qk == q) v = g.unit ? T(1) : tval(q, qk);
            }
            tv = v;
            const int kx = BT ? e / TS : e % TS, c = BT ? e % TS : e / TS;
            xv = (kx < K && c < C) ? *xaddr(k0 + kx, c0 + c) : T(0);
        };
        auto put = [&](int u, T tv, T xv) {
            const int e = tid + u * kTriThreads;
            sT[TT ? e % TS : e / TS][TT ? e / TS : e % TS] = tv;
            sX[BT ? e / TS : e % TS][BT ? e % TS : e / TS] = xv;
        };
        if (PREFETCH && kc_begin < kc_end) {
#pragma unroll
            for (int u = 0; u < EPR; ++u) chunk_vals(kc_begin, u, rt[u], rx[u]);
        }
        for (int kc = kc_begin; kc < kc_end; ++kc) {
            __syncthreads();   // the previous chunk's readers are done
            if (PREFETCH) {
#pragma unroll
                for (int u = 0; u < EPR; ++u) put(u, rt[u], rx[u]);
            } else {
                // all the chunk's loads before its shared-memory stores: interleaved, each
                // load would wait for the store before it (a generic pointer could alias it)
                constexpr int H = EPT / 2;   // in two halves: the registers stay under the solve's
#pragma unroll
                for (int u0 = 0; u0 < EPT; u0 += H) {
                    T tv[H], xv[H];
#pragma unroll
                    for (int u = 0; u < H; ++u) chunk_vals(kc, u0 + u, tv[u], xv[u]);
#pragma unroll
                    for (int u = 0; u < H; ++u) put(u0 + u, tv[u], xv[u]);
                }
            }
            __syncthreads();
            if (PREFETCH && kc + 1 < kc_end) {
#pragma unroll
                for (int u = 0; u < EPR; ++u) chunk_vals(kc + 1, u, rt[u], rx[u]);
            }
#pragma unroll 8
            for (int kk = 0; kk < TS; ++kk) {
                T ta[4], xb[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) ta[a] = sT[kk][tx + 8 * a];
#pragma unroll
                for (int b = 0; b < 4; ++b) xb[b] = sX[kk][ty * 4 + b];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b] = SOLVE ? fma(-ta[a], xb[b], acc[a][b])
                                                                  : fma(ta[a], xb[b], acc[a][b]);
            }
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) sS[tx + 8 * a][ty * 4 + b] = SOLVE ? acc[a][b] : g.alpha * acc[a][b];
        __syncthreads();   // sS and the diagonal block complete (the first tile has no chunk barrier)
        if (SOLVE && tid < TS) {
            rcp[tid] = T(1) / sD[tid][tid];
            __syncwarp();
            // lane = column: forward substitution through the diagonal block
            T s[TS];
#pragma unroll
            for (int r = 0; r < TS; ++r) s[r] = sS[r][tid];
#pragma unroll
            for (int r = 0; r < TS; ++r) {
                const T x = s[r] * rcp[r];
                sS[r][tid] = x;
#pragma unroll
                for (int r2 = r + 1; r2 < TS; ++r2) s[r2] = fma(-sD[r2][r], x, s[r2]);
            }
        }
        __syncthreads();
        for (int e = tid; e < TS * TS; e += kTriThreads) {
            const int r = BT ? e / TS : e % TS, c = BT ? e % TS : e / TS;
            if (r < R && c < C) *xaddr(q0 + r, c0 + c) = sS[r][c];
        }
        __syncthreads();
    }
}

template <typename T, bool S, bool F, bool TT, bool BT>
static void tri_launch(const TriArgs<T>& g, int panels, int batch, unsigned blocks, cudaStream_t s) {
    tri_panel_kernel<T, S, F, TT, BT><<<blocks, kTriThreads, 0, s>>>(g, panels, batch);
}

template <typename T>
static void tri_dispatch(int code, const TriArgs<T>& g, int panels, int batch, unsigned blocks, cudaStream_t s) {
#define MB200_TRI_CASE(c)                                                                                       \
    case c:                                                                                                     \
        tri_launch<T, ((c) & 8) != 0, ((c) & 4) != 0, ((c) & 2) != 0, ((c) & 1) != 0>(g, panels, batch, blocks, s); \
        break;
    switch (code) {
        MB200_TRI_CASE(0) MB200_TRI_CASE(1) MB200_TRI_CASE(2) MB200_TRI_CASE(3)
        MB200_TRI_CASE(4) MB200_TRI_CASE(5) MB200_TRI_CASE(6) MB200_TRI_CASE(7)
        MB200_TRI_CASE(8) MB200_TRI_CASE(9) MB200_TRI_CASE(10) MB200_TRI_CASE(11)
        MB200_TRI_CASE(12) MB200_TRI_CASE(13) MB200_TRI_CASE(14) MB200_TRI_CASE(15)
    }
#undef MB200_TRI_CASE
}

// The _max_nocheck body of both routines (magmablas/ztrmm_vbatched.cpp:31-32: quick
// return when max_m or max_n <= 0).
template <typename T>
static void tri_vbatched(bool solve, magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                         int* m, int* n, T alpha, T* const* A, int* lda, T** B, int* ldb, int batch, int max_m,
                         int max_n, magma_queue_t queue) {
    if (max_m <= 0 || max_n <= 0 || batch <= 0) return;
    const bool left = side == MagmaLeft, opt = transA != MagmaNoTrans;
    const bool op_lower = (uplo == MagmaLower) != opt;        // op(A) lower
    const bool t_lower = left ? op_lower : !op_lower;         // T = op(A) or op(A)^T
    const bool tt = left ? opt : !opt;                        // T(i,k) = A(k,i)
    const bool bt = !left;                                    // X = B^T
    const bool flip = solve ? !t_lower : t_lower;
    const int panels = ceildiv(left ? max_n : max_m, kTriTile);
    const long blocks = (long)batch * panels;
    if (blocks > 0x7fffffffL) {
        magma_xerbla(solve ? "magmablas_trsm_vbatched" : "magmablas_trmm_vbatched", 12);
        return;
    }
    const TriArgs<T> g{A, B, m, n, lda, ldb, 0, 0, 0, 0, alpha, left, diag == MagmaUnit};
    const int code = (solve ? 8 : 0) | (flip ? 4 : 0) | (tt ? 2 : 0) | (bt ? 1 : 0);
    tri_dispatch<T>(code, g, panels, batch, (unsigned)blocks, queue->stream);
}

// Fixed size (magmablas/ztrsm_batched.cpp:196-229, magmablas/ztrmm_batched_core.cu:811-832):
// side -1, uplo -2, transA -3, diag -4, m -5, n -6, ldda < max(1, rows of A) -9,
// lddb < max(1, m) -11; quick return when m or n is 0.
template <typename T>
static void tri_batched(bool solve, const char* name, magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,
                        magma_diag_t diag, int m, int n, T alpha, T* const* A, int lda, T** B, int ldb, int batch,
                        magma_queue_t queue) {
    int info = 0;
    const int nrow_a = side == MagmaLeft ? m : n;
    if (side != MagmaLeft && side != MagmaRight) info = -1;
    else if (uplo != MagmaUpper && uplo != MagmaLower) info = -2;
    else if (transA != MagmaNoTrans && transA != MagmaTrans && transA != MagmaConjTrans) info = -3;
    else if (diag != MagmaUnit && diag != MagmaNonUnit) info = -4;
    else if (m < 0) info = -5;
    else if (n < 0) info = -6;
    else if (lda < std::max(1, nrow_a)) info = -9;
    else if (ldb < std::max(1, m)) info = -11;
    if (info != 0) {
        magma_xerbla(name, -info);
        return;
    }
    if (m == 0 || n == 0 || batch <= 0) return;
    const bool left = side == MagmaLeft, opt = transA != MagmaNoTrans;
    const bool op_lower = (uplo == MagmaLower) != opt;
    const bool t_lower = left ? op_lower : !op_lower;
    const bool tt = left ? opt : !opt;
    const bool flip = solve ? !t_lower : t_lower;
    const int panels = ceildiv(left ? n : m, kTriTile);
    const long blocks = (long)batch * panels;
    if (blocks > 0x7fffffffL) {
        magma_xerbla(name, 12);
        return;
    }
    const TriArgs<T> g{A, B, nullptr, nullptr, nullptr, nullptr, m, n, lda, ldb, alpha, left, diag == MagmaUnit};
    const int code = (solve ? 8 : 0) | (flip ? 4 : 0) | (tt ? 2 : 0) | (!left ? 1 : 0);
    tri_dispatch<T>(code, g, panels, batch, (unsigned)blocks, queue->stream);
}

// magmablas/vbatched_check.cu:134-181 (trsm) and :785-833 (trmm): side -1, uplo -2,
// transA -3, diag -4, m -5, n -6, ldda < max(1, rows of A) -9, lddb < max(1, m) -11,
// batchCount -12. Fills the maxima of m and n.
static int tri_vbatched_check(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag, int* m,
                              int* n, int* lda, int* ldb, int batch, magma_queue_t queue, int mx[2]) {
    if (side != MagmaLeft && side != MagmaRight) return -1;
    if (uplo != MagmaUpper && uplo != MagmaLower) return -2;
    if (transA != MagmaNoTrans && transA != MagmaTrans && transA != MagmaConjTrans) return -3;
    if (diag != MagmaUnit && diag != MagmaNonUnit) return -4;
    if (batch < 0) return -12;
    mx[0] = mx[1] = 0;
    if (batch == 0) return 0;
    int r[6];
    if (reduce_sizes(m, n, nullptr, batch, queue, r)) return MAGMA_ERR_UNKNOWN;
    if (r[3] < 0) return -5;
    if (r[4] < 0) return -6;
    int sl = 0;
    if (ld_slack1(side == MagmaLeft ? m : n, lda, batch, queue, &sl)) return MAGMA_ERR_UNKNOWN;
    if (sl < 0) return -9;
    if (ld_slack1(m, ldb, batch, queue, &sl)) return MAGMA_ERR_UNKNOWN;
    if (sl < 0) return -11;
    mx[0] = r[0];
    mx[1] = r[1];
    return 0;
}

}  // namespace mb200

using namespace mb200;

#define MB200_TRI_API(P, T, OP, SOLVE)                                                                                \
    void magmablas_##P##OP##_vbatched_max_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,         \
                                                  magma_diag_t diag, magma_int_t* m, magma_int_t* n, T alpha,         \
                                                  T** dA_array, magma_int_t* ldda, T** dB_array, magma_int_t* lddb,   \
                                                  magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,       \
                                                  magma_queue_t queue) {                                              \
        tri_vbatched<T>(SOLVE, side, uplo, transA, diag, m, n, alpha, dA_array, ldda, dB_array, lddb, batchCount,    \
                        max_m, max_n, queue);                                                                         \
    }                                                                                                                 \
    void magmablas_##P##OP##_vbatched_max(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,                 \
                                          magma_diag_t diag, magma_int_t* m, magma_int_t* n, T alpha, T** dA_array,   \
                                          magma_int_t* ldda, T** dB_array, magma_int_t* lddb, magma_int_t batchCount, \
                                          magma_int_t max_m, magma_int_t max_n, magma_queue_t queue) {                \
        int mx[2];                                                                                                    \
        const int info = tri_vbatched_check(side, uplo, transA, diag, m, n, ldda, lddb, batchCount, queue, mx);      \
        if (info != 0) {                                                                                              \
            magma_xerbla(__func__, -info);                                                                            \
            return;                                                                                                   \
        }                                                                                                             \
        tri_vbatched<T>(SOLVE, side, uplo, transA, diag, m, n, alpha, dA_array, ldda, dB_array, lddb, batchCount,    \
                        max_m, max_n, queue);                                                                         \
    }                                                                                                                 \
    void magmablas_##P##OP##_vbatched_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,             \
                                              magma_diag_t diag, magma_int_t* m, magma_int_t* n, T alpha,             \
                                              T** dA_array, magma_int_t* ldda, T** dB_array, magma_int_t* lddb,       \
                                              magma_int_t batchCount, magma_queue_t queue) {                          \
        int r[6];                                                                                                     \
        if (batchCount <= 0 || reduce_sizes(m, n, nullptr, batchCount, queue, r)) return;                            \
        tri_vbatched<T>(SOLVE, side, uplo, transA, diag, m, n, alpha, dA_array, ldda, dB_array, lddb, batchCount,    \
                        r[0], r[1], queue);                                                                           \
    }                                                                                                                 \
    void magmablas_##P##OP##_vbatched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,  \
                                      magma_int_t* m, magma_int_t* n, T alpha, T** dA_array, magma_int_t* ldda,       \
                                      T** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_queue_t queue) { \
        int mx[2];                                                                                                    \
        const int info = tri_vbatched_check(side, uplo, transA, diag, m, n, ldda, lddb, batchCount, queue, mx);      \
        if (info != 0) {                                                                                              \
            magma_xerbla(__func__, -info);                                                                            \
            return;                                                                                                   \
        }                                                                                                             \
        tri_vbatched<T>(SOLVE, side, uplo, transA, diag, m, n, alpha, dA_array, ldda, dB_array, lddb, batchCount,    \
                        mx[0], mx[1], queue);                                                                         \
    }

#define MB200_TRI_FIXED_API(P, T, OP, SOLVE)                                                                          \
    void magmablas_##P##OP##_batched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,   \
                                     magma_int_t m, magma_int_t n, T alpha, T** dA_array, magma_int_t ldda,          \
                                     T** dB_array, magma_int_t lddb, magma_int_t batchCount, magma_queue_t queue) {  \
        tri_batched<T>(SOLVE, __func__, side, uplo, transA, diag, m, n, alpha, dA_array, ldda, dB_array, lddb,       \
                       batchCount, queue);                                                                            \
    }

extern "C" {
MB200_TRI_FIXED_API(d, double, trsm, true)
MB200_TRI_FIXED_API(s, float, trsm, true)
MB200_TRI_FIXED_API(d, double, trmm, false)
MB200_TRI_FIXED_API(s, float, trmm, false)
MB200_TRI_API(d, double, trsm, true)
MB200_TRI_API(s, float, trsm, true)
MB200_TRI_API(d, double, trmm, false)
MB200_TRI_API(s, float, trmm, false)
}
