// gemm.cu -- batched and variable-size batched GEMM: C = alpha op(A) op(B) + beta C.
//
// Replaces magmablas_{d,s}gemm_batched_core (magmablas/dgemm_batched_core.cu:161-436) and
// magmablas_{d,s}gemm_vbatched_core (magmablas/dgemm_vbatched_core.cu:28-266). One
// thread block computes one BM x BN tile of one instance's C (three CUDA-core tile
// shapes: 64x64 with 256 threads, 32x32 and 16x16 with 64 threads, and for FP64 a
// 64x64 tile on the tensor cores, gemm_dmma_kernel); op(A) and op(B) are
// staged through shared memory in K chunks of 16, transposed at load time so the
// inner loop always reads contiguous vectors, with the next chunk prefetched into
// registers while the current one is used. Every shape accumulates each output
// over K in the same order, so the shapes give bit-identical results. Variable-size
// batches are bucketed by max(M, N) on the device; each bucket runs the tile shape
// the tuning table names for it (tuning.h), on its own auxiliary stream, with
// (instance, tile) pairs along grid.x sized by the bucket's edge; tiles past an
// instance's own size exit at once.
// Epilogue as the reference (magmablas/gemm_template_device.cuh:197-227): C is not
// read when beta == 0. SYRK (C = alpha op(A) op(A)^T + beta C on one triangle) is the
// same kernel with B = A and the other transpose, tiles outside the triangle exiting
// at once and the epilogue writing only the triangle (the reference's herk template,
// magmablas/herk_template_kernel_vbatched.cuh, likewise skips those tiles).
#include "internal.h"
#include "vbatched.h"
#include "tuning.h"
#include "lu_sizes.h"
#include "tc_ptx.cuh"
#include <algorithm>

namespace mb200 {

struct GemmSizes {
    int m, n, k, lda, ldb, ldc;
    const int *m_arr, *n_arr, *k_arr, *lda_arr, *ldb_arr, *ldc_arr;
    int tri;   // 0: all of C; 1: lower triangle only (i >= j); 2: upper only (syrk)
    __device__ __forceinline__ int M(int i) const { return m_arr ? m_arr[i] : m; }
    __device__ __forceinline__ int N(int i) const { return n_arr ? n_arr[i] : n; }
    __device__ __forceinline__ int K(int i) const { return k_arr ? k_arr[i] : k; }
    __device__ __forceinline__ int LDA(int i) const { return lda_arr ? lda_arr[i] : lda; }
    __device__ __forceinline__ int LDB(int i) const { return ldb_arr ? ldb_arr[i] : ldb; }
    __device__ __forceinline__ int LDC(int i) const { return ldc_arr ? ldc_arr[i] : ldc; }
};

// One tile shape of the kernel: BM x BN tile of C, TM x TN outputs per thread.
template <int BM_, int BN_, int TM_, int TN_, int MINB_D_, int MINB_F_>
struct GemmTile {
    // MINB_D / MINB_F: resident blocks per SM the FP64 / FP32 register allocations are sized for
    static constexpr int BM = BM_, BN = BN_, BK = 16, TM = TM_, TN = TN_, MINB_D = MINB_D_, MINB_F = MINB_F_;
    static constexpr int NT = (BM / TM) * (BN / TN);
    static constexpr int EA = BM * BK / NT, EB = BK * BN / NT;   // staged elements per thread
};
// The variants the tuning table chooses between (index = variant id).
using GemmTile0 = GemmTile<64, 64, 4, 4, 2, 3>;     // 256 threads
using GemmTile1 = GemmTile<32, 32, 4, 4, 10, 16>;   // 64 threads
using GemmTile2 = GemmTile<16, 16, 2, 2, 16, 16>;   // 64 threads

// C = alpha acc + beta C for a thread's TM x TN outputs (rows tx + (BM/TM) i, columns
// ty TN + j of the tile). Every read of C goes out before the first write: interleaved,
// each read would wait for the previous write (the compiler cannot rule out aliasing).
template <typename T, int BM, int TM, int TN>
__device__ __forceinline__ void gemm_tile_epilogue(const GemmSizes& g, T alpha, T beta, T* C, int ldc, int m, int n,
                                                   int i0, int j0, int tx, int ty, const T (&acc)[TM][TN]) {
    T cv[TM][TN];
    bool in[TM][TN];
#pragma unroll
    for (int j = 0; j < TN; ++j) {
        const int gj = j0 + ty * TN + j;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int gi = i0 + tx + (BM / TM) * i;
            in[i][j] = gj < n && gi < m && !(g.tri == 1 && gj > gi) && !(g.tri == 2 && gi > gj);
            cv[i][j] = (in[i][j] && beta != T(0)) ? C[gi + (size_t)gj * ldc] : T(0);
        }
    }
#pragma unroll
    for (int j = 0; j < TN; ++j) {
        const int gj = j0 + ty * TN + j;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int gi = i0 + tx + (BM / TM) * i;
            if (in[i][j])
                C[gi + (size_t)gj * ldc] = (beta == T(0)) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * cv[i][j];
        }
    }
}

template <typename T, bool TA, bool TB, typename S>
__global__ void __launch_bounds__(S::NT, (sizeof(T) == 8 ? S::MINB_D : S::MINB_F))
gemm_tile_kernel(GemmSizes g, T alpha, const T* const* __restrict__ A_arr, const T* const* __restrict__ B_arr, T beta,
                 T** __restrict__ C_arr, int tiles_m, int tiles_n, WorkList wl) {
    constexpr int BM = S::BM, BN = S::BN, BK = S::BK, TM = S::TM, TN = S::TN, NT = S::NT;
    constexpr int EA = S::EA, EB = S::EB;
    // rows padded by one element: the K-fastest staging stores would otherwise
    // hit one bank 16 times
    __shared__ T sA[BK][BM + 1];
    __shared__ T sB[BK][BN + 1];
    const int tiles = tiles_m * tiles_n;
    const int w = blockIdx.x / tiles;
    if (w >= wl.size()) return;
    const int id = wl.at(w);
    const int t = blockIdx.x - w * tiles;
    const int i0 = (t / tiles_n) * BM, j0 = (t % tiles_n) * BN;
    const int m = g.M(id), n = g.N(id), k = g.K(id);
    if (i0 >= m || j0 >= n) return;
    if ((g.tri == 1 && j0 > i0 + BM - 1) || (g.tri == 2 && i0 > j0 + BN - 1)) return;   // tile outside the triangle
    const int lda = g.LDA(id), ldb = g.LDB(id), ldc = g.LDC(id);
    const T* A = A_arr[id];
    const T* B = B_arr[id];
    T* C = C_arr[id];
    const int tid = threadIdx.x;
    // thread (tx, ty) owns rows tx + 16*i and columns ty*4 + j of the tile: consecutive
    // threads read consecutive A values (no bank conflicts) and write consecutive
    // rows of column-major C (coalesced); the B values are warp-wide broadcasts
    const int tx = tid % (BM / TM), ty = tid / (BM / TM);
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

    // each thread stages EA elements of the A chunk and EB of the B chunk
    T ra[EA], rb[EB];
    auto load_chunk = [&](int k0) {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            const int idx = tid + e * NT;
            int r, c;
            if (!TA) { r = idx % BM; c = idx / BM; } else { c = idx % BK; r = idx / BK; }
            const int gi = i0 + r, gk = k0 + c;
            ra[e] = (gi < m && gk < k) ? (TA ? A[gk + (size_t)gi * lda] : A[gi + (size_t)gk * lda]) : T(0);
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            const int idx = tid + e * NT;
            int c, j;
            if (!TB) { c = idx % BK; j = idx / BK; } else { j = idx % BN; c = idx / BN; }
            const int gk = k0 + c, gj = j0 + j;
            rb[e] = (gk < k && gj < n) ? (TB ? B[gj + (size_t)gk * ldb] : B[gk + (size_t)gj * ldb]) : T(0);
        }
    };
    auto store_chunk = [&]() {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            const int idx = tid + e * NT;
            int r, c;
            if (!TA) { r = idx % BM; c = idx / BM; } else { c = idx % BK; r = idx / BK; }
            sA[c][r] = ra[e];
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            const int idx = tid + e * NT;
            int c, j;
            if (!TB) { c = idx % BK; j = idx / BK; } else { j = idx % BN; c = idx / BN; }
            sB[c][j] = rb[e];
        }
    };
    if (k > 0) load_chunk(0);
    for (int k0 = 0; k0 < k; k0 += BK) {
        __syncthreads();
        store_chunk();
        __syncthreads();
        if (k0 + BK < k) load_chunk(k0 + BK);   // prefetch the next chunk while computing
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = sA[kk][tx + (BM / TM) * i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = sB[kk][ty * TN + j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
    }
    gemm_tile_epilogue<T, BM, TM, TN>(g, alpha, beta, C, ldc, m, n, i0, j0, tx, ty, acc);
}

// NN form of the CUDA-core tiles with an asynchronous operand pipeline: each K chunk
// of op(A) and op(B) is copied global -> shared by cp.async (element-sized copies,
// zero-filled past the instance's edges), three chunks in flight, so the loads of
// chunks c+1 and c+2 overlap the arithmetic of chunk c without passing through
// registers. The staged layout and the inner loop are gemm_tile_kernel's, so each
// output receives the same fma's in the same order (bit-identical variants).
template <int STAGES, typename T, typename S>
struct GemmAsyncSmem {
    T a[STAGES][S::BK][S::BM + 1];
    T b[STAGES][S::BK][S::BN + 1];
};

__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, bool valid, int bytes) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    const int sz = valid ? bytes : 0;   // src-size 0: the destination is zero-filled, nothing is read
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(sz) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(sz) : "memory");
}

template <typename T, typename S>
__global__ void __launch_bounds__(S::NT, (sizeof(T) == 8 ? S::MINB_D : S::MINB_F))
gemm_async_kernel(GemmSizes g, T alpha, const T* const* __restrict__ A_arr, const T* const* __restrict__ B_arr,
                  T beta, T** __restrict__ C_arr, int tiles_m, int tiles_n, WorkList wl) {
    constexpr int BM = S::BM, BN = S::BN, BK = S::BK, TM = S::TM, TN = S::TN, NT = S::NT, ST = 3;
    constexpr int EA = S::EA, EB = S::EB;
    extern __shared__ __align__(16) unsigned char gemm_async_raw[];
    GemmAsyncSmem<ST, T, S>& sm = *reinterpret_cast<GemmAsyncSmem<ST, T, S>*>(gemm_async_raw);
    const int tiles = tiles_m * tiles_n;
    const int w = blockIdx.x / tiles;
    if (w >= wl.size()) return;
    const int id = wl.at(w);
    const int t = blockIdx.x - w * tiles;
    const int i0 = (t / tiles_n) * BM, j0 = (t % tiles_n) * BN;
    const int m = g.M(id), n = g.N(id), k = g.K(id);
    if (i0 >= m || j0 >= n) return;
    if ((g.tri == 1 && j0 > i0 + BM - 1) || (g.tri == 2 && i0 > j0 + BN - 1)) return;
    const int lda = g.LDA(id), ldb = g.LDB(id), ldc = g.LDC(id);
    const T* A = A_arr[id];
    const T* B = B_arr[id];
    T* C = C_arr[id];
    const int tid = threadIdx.x;
    const int tx = tid % (BM / TM), ty = tid / (BM / TM);
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
    auto issue = [&](int chunk) {
        const int st = chunk % ST, k0 = chunk * BK;
#pragma unroll
        for (int e = 0; e < EA; ++e) {   // A (M x K, column-major): rows fastest, contiguous
            const int idx = tid + e * NT, r = idx % BM, c = idx / BM;
            const bool v = (i0 + r < m) && (k0 + c < k);
            cp_async_elem(&sm.a[st][c][r], v ? A + (i0 + r) + (size_t)(k0 + c) * lda : A, v, sizeof(T));
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {   // B (K x N, column-major): k fastest, contiguous
            const int idx = tid + e * NT, c = idx % BK, j = idx / BK;
            const bool v = (k0 + c < k) && (j0 + j < n);
            cp_async_elem(&sm.b[st][c][j], v ? B + (k0 + c) + (size_t)(j0 + j) * ldb : B, v, sizeof(T));
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int nchunks = (k + BK - 1) / BK;
    issue(0);
    if (nchunks > 1) issue(1); else asm volatile("cp.async.commit_group;" ::: "memory");
    for (int c = 0; c < nchunks; ++c) {
        asm volatile("cp.async.wait_group 1;" ::: "memory");   // chunk c has landed (c+1 may be in flight)
        __syncthreads();                                         // ... for every thread; stage (c+2)%3 is free
        if (c + 2 < nchunks) issue(c + 2); else asm volatile("cp.async.commit_group;" ::: "memory");
        const int st = c % ST;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = sm.a[st][kk][tx + (BM / TM) * i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = sm.b[st][kk][ty * TN + j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    gemm_tile_epilogue<T, BM, TM, TN>(g, alpha, beta, C, ldc, m, n, i0, j0, tx, ty, acc);
}

// FP64 tile on the tensor cores (variant 3): a 64x64 tile of C per 256-thread block,
// each warp a 32x16 sub-tile as 4x2 tiles of 8x8 updated by mma.sync m8n8k4 .f64.
// Staging is that of gemm_tile_kernel (K chunks of 16, transposed at load time, the
// next chunk prefetched into registers); the fragments are read from the staged
// chunk (rows padded to 68 doubles: the four k rows a fragment load touches fall on
// different banks). An m8n8k4 FP64 MMA applies its four products to each element as
// fma's in ascending k, and the k-steps run in ascending order, so every output gets
// exactly the fma chain of the CUDA-core tiles: the variants stay bit-identical.
__device__ __forceinline__ void gemm_dmma(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(256, 2)
gemm_dmma_kernel(GemmSizes g, double alpha, const double* const* __restrict__ A_arr,
                 const double* const* __restrict__ B_arr, double beta, double** __restrict__ C_arr, int tiles_m,
                 int tiles_n, WorkList wl) {
    constexpr int BM = 64, BN = 64, BK = 16, NT = 256, PAD = 68;
    constexpr int EA = BM * BK / NT, EB = BK * BN / NT;
    __shared__ __align__(16) double sA[BK][PAD];
    __shared__ __align__(16) double sB[BK][PAD];
    const int tiles = tiles_m * tiles_n;
    const int w = blockIdx.x / tiles;
    if (w >= wl.size()) return;
    const int id = wl.at(w);
    const int t = blockIdx.x - w * tiles;
    const int i0 = (t / tiles_n) * BM, j0 = (t % tiles_n) * BN;
    const int m = g.M(id), n = g.N(id), k = g.K(id);
    if (i0 >= m || j0 >= n) return;
    if ((g.tri == 1 && j0 > i0 + BM - 1) || (g.tri == 2 && i0 > j0 + BN - 1)) return;
    const int lda = g.LDA(id), ldb = g.LDB(id), ldc = g.LDC(id);
    const double* A = A_arr[id];
    const double* B = B_arr[id];
    double* C = C_arr[id];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;   // warp's sub-tile
    const int q = lane & 3, r8 = lane >> 2;
    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    double ra[EA], rb[EB];
    auto load_chunk = [&](int k0) {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            const int idx = tid + e * NT;
            int r, c;
            if (!TA) { r = idx % BM; c = idx / BM; } else { c = idx % BK; r = idx / BK; }
            const int gi = i0 + r, gk = k0 + c;
            ra[e] = (gi < m && gk < k) ? (TA ? A[gk + (size_t)gi * lda] : A[gi + (size_t)gk * lda]) : 0.0;
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            const int idx = tid + e * NT;
            int c, j;
            if (!TB) { c = idx % BK; j = idx / BK; } else { j = idx % BN; c = idx / BN; }
            const int gk = k0 + c, gj = j0 + j;
            rb[e] = (gk < k && gj < n) ? (TB ? B[gj + (size_t)gk * ldb] : B[gk + (size_t)gj * ldb]) : 0.0;
        }
    };
    auto store_chunk = [&]() {
#pragma unroll
        for (int e = 0; e < EA; ++e) {
            const int idx = tid + e * NT;
            int r, c;
            if (!TA) { r = idx % BM; c = idx / BM; } else { c = idx % BK; r = idx / BK; }
            sA[c][r] = ra[e];
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {
            const int idx = tid + e * NT;
            int c, j;
            if (!TB) { c = idx % BK; j = idx / BK; } else { j = idx % BN; c = idx / BN; }
            sB[c][j] = rb[e];
        }
    };
    if (k > 0) load_chunk(0);
    for (int k0 = 0; k0 < k; k0 += BK) {
        __syncthreads();
        store_chunk();
        __syncthreads();
        if (k0 + BK < k) load_chunk(k0 + BK);   // prefetch the next chunk while computing
#pragma unroll
        for (int s4 = 0; s4 < BK / 4; ++s4) {
            double af[4], bf[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = sA[4 * s4 + q][wm + 8 * i + r8];
#pragma unroll
            for (int j = 0; j < 2; ++j) bf[j] = sB[4 * s4 + q][wn + 8 * j + r8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) gemm_dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    // every read of C before the first write (as gemm_tile_epilogue)
    double cv[4][2][2];
    bool in[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gi = i0 + wm + 8 * i + r8;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = j0 + wn + 8 * j + 2 * q + h;
                in[i][j][h] = gi < m && gj < n && !(g.tri == 1 && gj > gi) && !(g.tri == 2 && gi > gj);
                cv[i][j][h] = (in[i][j][h] && beta != 0.0) ? C[gi + (size_t)gj * ldc] : 0.0;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gi = i0 + wm + 8 * i + r8;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = j0 + wn + 8 * j + 2 * q + h;
                if (in[i][j][h])
                    C[gi + (size_t)gj * ldc] =
                        (beta == 0.0) ? alpha * acc[i][j][h] : alpha * acc[i][j][h] + beta * cv[i][j][h];
            }
        }
    }
}

// FP32 tile on the tcgen05 tensor cores (FP32 variant 3): a 128x128 tile of C per
// 128-thread block, accumulated in tensor memory (128 lanes x 128 FP32 columns; thread t
// owns lane t = row t of the tile). K runs in chunks of 32: the threads stage op(A) and
// op(B) as split TF32 pairs (hi = x rounded to TF32, lo = x - hi) in the no-swizzle K-major
// layout of 8x4 core matrices, then one thread issues the chunk's four K = 8 steps as three
// MMAs each (lo*hi, hi*lo, hi*hi: ~21-bit products accumulated in FP32, the lo*lo term
// dropped) and commits them to an mbarrier the block waits on, bounded. Thread t stages
// row t of op(A) and of op(B)^T, its 32 loads issued together. B is staged for N rounded
// up to 16 columns (the MMA's N), zero past N; rows of A past M are left as they are (they
// only reach accumulator rows that are never stored); the K tail is zero in both operands.
// Unlike the CUDA-core tiles this is not the same fma chain: the results differ in the
// last bits and are held to the reference tester's bound
// ||C - C_ref|| / (sqrt(k+2) |alpha| ||A|| ||B|| + 2 |beta| ||C||) < 30 eps
// (testing/testing_sgemm_vbatched.cpp). A wait that runs out (about a second) leaves the
// tensor cores alone: the block computes its tile again on the CUDA cores instead.
constexpr int kTcGemmKc = 32;
constexpr long long kTcGemmWaitCycles = 2000000000LL;

__device__ __forceinline__ int tc_kmajor(int row, int k) {   // float index of (row, k) in a 32-wide K chunk
    return (((row >> 3) * 8 + (k >> 2)) * 8 + (row & 7)) * 4 + (k & 3);
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(128, 3)
gemm_tc_kernel(GemmSizes g, float alpha, const float* const* __restrict__ A_arr,
               const float* const* __restrict__ B_arr, float beta, float** __restrict__ C_arr, int tiles_m,
               int tiles_n, WorkList wl) {
    constexpr int BM = 128, BN = 128, KC = kTcGemmKc;
    extern __shared__ __align__(1024) unsigned char gemm_tc_smem[];
    float* sA = reinterpret_cast<float*>(gemm_tc_smem);   // [hi, lo][BM * KC]
    float* sB = sA + 2 * BM * KC;                          // [hi, lo][BN * KC]
    __shared__ unsigned long long mbar_word;
    __shared__ uint32_t tmem_base;
    const int tiles = tiles_m * tiles_n;
    const int w = blockIdx.x / tiles;
    if (w >= wl.size()) return;
    const int id = wl.at(w);
    const int tt = blockIdx.x - w * tiles;
    const int i0 = (tt / tiles_n) * BM, j0 = (tt % tiles_n) * BN;
    const int m = g.M(id), n = g.N(id), k = g.K(id);
    if (i0 >= m || j0 >= n) return;
    if ((g.tri == 1 && j0 > i0 + BM - 1) || (g.tri == 2 && i0 > j0 + BN - 1)) return;
    const int lda = g.LDA(id), ldb = g.LDB(id), ldc = g.LDC(id);
    const float* A = A_arr[id];
    const float* B = B_arr[id];
    float* C = C_arr[id];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int mrows = min(BM, m - i0), ncols = min(BN, n - j0);
    const int npad = (ncols + 15) & ~15;
    const uint32_t mbar = tc::smem_addr(&mbar_word);
    if (warp == 0) {
        tc::tmem_alloc(tc::smem_addr(&tmem_base), BN);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = tmem_base;
    const uint32_t idesc = tc::idesc_tf32(BM, npad, false);
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < k; k0 += KC) {
        // thread t stages row t of op(A) (rows < mrows) and row t of the N x K operand
        // op(B)^T (rows < npad): 32 values of the chunk each, all loads issued before
        // any is used, zero past K (and past N for B); rows of A past M stay unwritten
        float xa[KC], xb[KC];
        const int gi = i0 + tid, gj = j0 + tid;
#pragma unroll
        for (int q = 0; q < KC; ++q) {
            const int gk = k0 + q;
            xa[q] = (tid < mrows && gk < k) ? (TA ? A[gk + (size_t)gi * lda] : A[gi + (size_t)gk * lda]) : 0.0f;
            xb[q] = (tid < ncols && gk < k) ? (TB ? B[gj + (size_t)gk * ldb] : B[gk + (size_t)gj * ldb]) : 0.0f;
        }
        if (tid < mrows) {
#pragma unroll
            for (int q = 0; q < KC; q += 4) {
                float4 h, l;
                tc::split_tf32(xa[q], h.x, l.x);
                tc::split_tf32(xa[q + 1], h.y, l.y);
                tc::split_tf32(xa[q + 2], h.z, l.z);
                tc::split_tf32(xa[q + 3], h.w, l.w);
                *reinterpret_cast<float4*>(sA + tc_kmajor(tid, q)) = h;
                *reinterpret_cast<float4*>(sA + BM * KC + tc_kmajor(tid, q)) = l;
            }
        }
        if (tid < npad) {
#pragma unroll
            for (int q = 0; q < KC; q += 4) {
                float4 h, l;
                tc::split_tf32(xb[q], h.x, l.x);
                tc::split_tf32(xb[q + 1], h.y, l.y);
                tc::split_tf32(xb[q + 2], h.z, l.z);
                tc::split_tf32(xb[q + 3], h.w, l.w);
                *reinterpret_cast<float4*>(sB + tc_kmajor(tid, q)) = h;
                *reinterpret_cast<float4*>(sB + BN * KC + tc_kmajor(tid, q)) = l;
            }
        }
        tc::fence_proxy_async_smem();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int s4 = 0; s4 < KC / 8; ++s4) {   // K = 8 per MMA: two core matrices
                const uint64_t ah = tc::smem_desc(tc::smem_addr(sA + s4 * 64), 128, 1024);
                const uint64_t al = tc::smem_desc(tc::smem_addr(sA + BM * KC + s4 * 64), 128, 1024);
                const uint64_t bh = tc::smem_desc(tc::smem_addr(sB + s4 * 64), 128, 1024);
                const uint64_t bl = tc::smem_desc(tc::smem_addr(sB + BN * KC + s4 * 64), 128, 1024);
                tc::mma_tf32(tbase, al, bh, idesc, k0 > 0 || s4 > 0);
                tc::mma_tf32(tbase, ah, bl, idesc, true);
                tc::mma_tf32(tbase, ah, bh, idesc, true);
            }
            tc::commit(mbar);
        }
        bool done = false;
        const long long t0 = clock64();
        while (!(done = tc::mbar_try_wait(mbar, phase)) && clock64() - t0 < kTcGemmWaitCycles) {
        }
        phase ^= 1u;
        if (__syncthreads_or(!done)) {   // every thread leaves the loop for the CUDA-core path below
            ok = false;
            break;
        }
        tc::fence_after_sync();
    }
    if (!ok && tid < mrows) {
        // the tensor cores did not answer in time: row tid of the tile from global memory
        // with FP32 fma's (slow, but the tile is right)
        const int gi = i0 + tid;
        for (int c = 0; c < ncols; ++c) {
            const int gj = j0 + c;
            if ((g.tri == 1 && gj > gi) || (g.tri == 2 && gi > gj)) continue;
            float acc = 0.0f;
            for (int kk = 0; kk < k; ++kk) {
                const float a = TA ? A[kk + (size_t)gi * lda] : A[gi + (size_t)kk * lda];
                const float b = TB ? B[gj + (size_t)kk * ldb] : B[kk + (size_t)gj * ldb];
                acc = fmaf(a, b, acc);
            }
            float* cp = C + gi + (size_t)gj * ldc;
            *cp = (beta == 0.0f) ? alpha * acc : alpha * acc + beta * (*cp);
        }
    }
    if (ok) {
        const int gi = i0 + tid;
        const uint32_t trow = tbase + (uint32_t(32 * warp) << 16);
        for (int c0 = 0; c0 < ncols; c0 += 32) {
            float v[32];
            if (k > 0) {
                tc::tmem_ld32(trow + uint32_t(c0), v);
                tc::wait_ld();
            } else {
#pragma unroll
                for (int c = 0; c < 32; ++c) v[c] = 0.0f;
            }
            if (tid < mrows) {
                // all 32 reads of C before any write (the writes could alias later reads, so
                // interleaved they would wait for each other)
                float cv[32];
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int gj = j0 + c0 + c;
                    const bool in = c0 + c < ncols && !(g.tri == 1 && gj > gi) && !(g.tri == 2 && gi > gj);
                    cv[c] = (in && beta != 0.0f) ? C[gi + (size_t)gj * ldc] : 0.0f;
                }
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int gj = j0 + c0 + c;
                    if (c0 + c >= ncols || (g.tri == 1 && gj > gi) || (g.tri == 2 && gi > gj)) continue;
                    C[gi + (size_t)gj * ldc] = (beta == 0.0f) ? alpha * v[c] : alpha * v[c] + beta * cv[c];
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tbase, BN);
}

constexpr int kTcGemmSmem = 4 * 128 * kTcGemmKc * (int)sizeof(float);   // A and B, hi and lo

template <typename T>
static magma_int_t gemm_launch_tc(bool TA, bool TB, const GemmSizes& g, T alpha, const T* const* A, const T* const* B,
                                  T beta, T** C, const WorkList& wl, int bound, int max_m, int max_n, cudaStream_t s) {
    if constexpr (sizeof(T) != 4) {
        return MAGMA_ERR_NOT_SUPPORTED;
    } else {
        const int tiles_m = ceildiv(max_m, 128), tiles_n = ceildiv(max_n, 128);
        const long blocks = (long)bound * tiles_m * tiles_n;
        if (blocks > 0x7fffffffL) return MAGMA_ERR_NOT_SUPPORTED;
        const dim3 grid((unsigned)blocks);
        auto launch = [&](auto kern) {
            ensure_dynamic_smem((const void*)kern, kTcGemmSmem);
            kern<<<grid, 128, kTcGemmSmem, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
        };
        if (!TA && !TB) launch(gemm_tc_kernel<false, false>);
        else if (!TA && TB) launch(gemm_tc_kernel<false, true>);
        else if (TA && !TB) launch(gemm_tc_kernel<true, false>);
        else launch(gemm_tc_kernel<true, true>);
        return 0;
    }
}

// NN form of the FP64 tensor-core tile fed by the cp.async pipeline of gemm_async_kernel:
// three K chunks of 16 in flight (element-sized copies, zero-filled past the edges) into
// rows padded to 68 doubles, the same fragments, k-steps and epilogue as gemm_dmma_kernel,
// so the same bits.
#ifndef MB200_DMMA_WARP_N
#define MB200_DMMA_WARP_N 32
#endif
constexpr int kDmmaWarpN = MB200_DMMA_WARP_N;
struct GemmDmmaAsyncSmem {
    double a[3][16][68];
    double b[3][16][68];
};

// WN: each warp's tile is 32 x WN (4 x WN/8 tiles of 8x8); 64 x 64 / (32 WN) warps.
template <int WN>
__global__ void __launch_bounds__(64 * 64 / (32 * WN) * 32, (WN == 16 ? 2 : 3))
gemm_dmma_async_kernel(GemmSizes g, double alpha, const double* const* __restrict__ A_arr,
                       const double* const* __restrict__ B_arr, double beta, double** __restrict__ C_arr,
                       int tiles_m, int tiles_n, WorkList wl) {
    constexpr int BM = 64, BN = 64, BK = 16, NT = 64 * 64 / (32 * WN) * 32, ST = 3, TJ = WN / 8;
    constexpr int EA = BM * BK / NT, EB = BK * BN / NT;
    extern __shared__ __align__(16) unsigned char gemm_dmma_async_raw[];
    GemmDmmaAsyncSmem& sm = *reinterpret_cast<GemmDmmaAsyncSmem*>(gemm_dmma_async_raw);
    const int tiles = tiles_m * tiles_n;
    const int w = blockIdx.x / tiles;
    if (w >= wl.size()) return;
    const int id = wl.at(w);
    const int t = blockIdx.x - w * tiles;
    const int i0 = (t / tiles_n) * BM, j0 = (t % tiles_n) * BN;
    const int m = g.M(id), n = g.N(id), k = g.K(id);
    if (i0 >= m || j0 >= n) return;
    if ((g.tri == 1 && j0 > i0 + BM - 1) || (g.tri == 2 && i0 > j0 + BN - 1)) return;
    const int lda = g.LDA(id), ldb = g.LDB(id), ldc = g.LDC(id);
    const double* A = A_arr[id];
    const double* B = B_arr[id];
    double* C = C_arr[id];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * WN;   // warp's sub-tile
    const int q = lane & 3, r8 = lane >> 2;
    double acc[4][TJ][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < TJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    auto issue = [&](int chunk) {
        const int st = chunk % ST, k0 = chunk * BK;
#pragma unroll
        for (int e = 0; e < EA; ++e) {   // A (M x K, column-major): rows fastest, contiguous
            const int idx = tid + e * NT, r = idx % BM, c = idx / BM;
            const bool v = (i0 + r < m) && (k0 + c < k);
            cp_async_elem(&sm.a[st][c][r], v ? A + (i0 + r) + (size_t)(k0 + c) * lda : A, v, 8);
        }
#pragma unroll
        for (int e = 0; e < EB; ++e) {   // B (K x N, column-major): k fastest, contiguous
            const int idx = tid + e * NT, c = idx % BK, j = idx / BK;
            const bool v = (k0 + c < k) && (j0 + j < n);
            cp_async_elem(&sm.b[st][c][j], v ? B + (k0 + c) + (size_t)(j0 + j) * ldb : B, v, 8);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int nchunks = (k + BK - 1) / BK;
    if (nchunks > 0) issue(0);
    if (nchunks > 1) issue(1); else asm volatile("cp.async.commit_group;" ::: "memory");
    for (int c = 0; c < nchunks; ++c) {
        asm volatile("cp.async.wait_group 1;" ::: "memory");   // chunk c has landed (c+1 may be in flight)
        __syncthreads();                                         // ... for every thread; stage (c+2)%3 is free
        if (c + 2 < nchunks) issue(c + 2); else asm volatile("cp.async.commit_group;" ::: "memory");
        const int st = c % ST;
#pragma unroll
        for (int s4 = 0; s4 < BK / 4; ++s4) {
            double af[4], bf[TJ];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = sm.a[st][4 * s4 + q][wm + 8 * i + r8];
#pragma unroll
            for (int j = 0; j < TJ; ++j) bf[j] = sm.b[st][4 * s4 + q][wn + 8 * j + r8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < TJ; ++j) gemm_dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // every read of C before the first write (as gemm_tile_epilogue)
    double cv[4][TJ][2];
    bool in[4][TJ][2];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gi = i0 + wm + 8 * i + r8;
#pragma unroll
        for (int j = 0; j < TJ; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = j0 + wn + 8 * j + 2 * q + h;
                in[i][j][h] = gi < m && gj < n && !(g.tri == 1 && gj > gi) && !(g.tri == 2 && gi > gj);
                cv[i][j][h] = (in[i][j][h] && beta != 0.0) ? C[gi + (size_t)gj * ldc] : 0.0;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gi = i0 + wm + 8 * i + r8;
#pragma unroll
        for (int j = 0; j < TJ; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gj = j0 + wn + 8 * j + 2 * q + h;
                if (in[i][j][h])
                    C[gi + (size_t)gj * ldc] =
                        (beta == 0.0) ? alpha * acc[i][j][h] : alpha * acc[i][j][h] + beta * cv[i][j][h];
            }
        }
    }
}

template <typename T>
static magma_int_t gemm_launch_dmma(bool TA, bool TB, const GemmSizes& g, T alpha, const T* const* A,
                                    const T* const* B, T beta, T** C, const WorkList& wl, int bound, int max_m,
                                    int max_n, cudaStream_t s) {
    if constexpr (sizeof(T) != 8) {
        return MAGMA_ERR_NOT_SUPPORTED;
    } else {
        const int tiles_m = ceildiv(max_m, 64), tiles_n = ceildiv(max_n, 64);
        const long blocks = (long)bound * tiles_m * tiles_n;
        if (blocks > 0x7fffffffL) return MAGMA_ERR_NOT_SUPPORTED;
        const dim3 grid((unsigned)blocks);
        if (!TA && !TB) {   // NN: the cp.async-fed form
            constexpr int WN = kDmmaWarpN;
            auto kern = gemm_dmma_async_kernel<WN>;
            const int smem = (int)sizeof(GemmDmmaAsyncSmem);
            ensure_dynamic_smem((const void*)kern, smem);
            kern<<<grid, 64 * 64 / (32 * WN) * 32, smem, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
        }
        else if (!TA && TB) gemm_dmma_kernel<false, true><<<grid, 256, 0, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
        else if (TA && !TB) gemm_dmma_kernel<true, false><<<grid, 256, 0, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
        else gemm_dmma_kernel<true, true><<<grid, 256, 0, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
        return 0;
    }
}

template <typename T, typename S>
static magma_int_t gemm_launch_tile(bool TA, bool TB, const GemmSizes& g, T alpha, const T* const* A, const T* const* B,
                                    T beta, T** C, const WorkList& wl, int bound, int max_m, int max_n,
                                    cudaStream_t s) {
    const int tiles_m = ceildiv(max_m, S::BM), tiles_n = ceildiv(max_n, S::BN);
    const long blocks = (long)bound * tiles_m * tiles_n;
    if (blocks > 0x7fffffffL) return MAGMA_ERR_NOT_SUPPORTED;
    const dim3 grid((unsigned)blocks);
    if (!TA && !TB && sizeof(T) == 8) {   // FP64 NN: the asynchronous-copy pipeline (measured faster
                                          // for FP64 on the C2 mix, slower for FP32)
        auto kern = gemm_async_kernel<T, S>;
        const int smem = (int)sizeof(GemmAsyncSmem<3, T, S>);
        ensure_dynamic_smem((const void*)kern, smem);
        kern<<<grid, S::NT, smem, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
    } else if (!TA && !TB) gemm_tile_kernel<T, false, false, S><<<grid, S::NT, 0, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
    else if (!TA && TB) gemm_tile_kernel<T, false, true, S><<<grid, S::NT, 0, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
    else if (TA && !TB) gemm_tile_kernel<T, true, false, S><<<grid, S::NT, 0, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
    else gemm_tile_kernel<T, true, true, S><<<grid, S::NT, 0, s>>>(g, alpha, A, B, beta, C, tiles_m, tiles_n, wl);
    return 0;
}

template <typename T>
static magma_int_t gemm_launch_variant(int variant, magma_trans_t ta, magma_trans_t tb, const GemmSizes& g, T alpha,
                                       const T* const* A, const T* const* B, T beta, T** C, const WorkList& wl,
                                       int bound, int max_m, int max_n, cudaStream_t s) {
    const bool TA = (ta != MagmaNoTrans), TB = (tb != MagmaNoTrans);   // real types: ConjTrans == Trans
    switch (variant) {
        case 1: return gemm_launch_tile<T, GemmTile1>(TA, TB, g, alpha, A, B, beta, C, wl, bound, max_m, max_n, s);
        case 2: return gemm_launch_tile<T, GemmTile2>(TA, TB, g, alpha, A, B, beta, C, wl, bound, max_m, max_n, s);
        case 3:   // the tensor cores: FP64 mma.sync (DMMA) tile, FP32 tcgen05 split-TF32 tile
            if (sizeof(T) == 8) return gemm_launch_dmma<T>(TA, TB, g, alpha, A, B, beta, C, wl, bound, max_m, max_n, s);
            return gemm_launch_tc<T>(TA, TB, g, alpha, A, B, beta, C, wl, bound, max_m, max_n, s);
        default: return gemm_launch_tile<T, GemmTile0>(TA, TB, g, alpha, A, B, beta, C, wl, bound, max_m, max_n, s);
    }
}

// Size buckets of max(M, N): the tuning table names a tile variant per bucket.
static const int kGemmEdges[kGemmBuckets] = {16, 32, 64, 1 << 30};

static int gemm_bucket_of(int mn) {
    for (int b = 0; b < kGemmBuckets; ++b)
        if (mn <= kGemmEdges[b]) return b;
    return kGemmBuckets - 1;
}

// Fixed size: one launch with the bucket's variant.
template <typename T>
static magma_int_t gemm_launch(magma_trans_t ta, magma_trans_t tb, const GemmSizes& g, T alpha, const T* const* A,
                               const T* const* B, T beta, T** C, int batch, int max_m, int max_n, cudaStream_t s) {
    const int v = tuning().gemm_variant[sizeof(T) == 8 ? 0 : 1][gemm_bucket_of(std::max(max_m, max_n))];
    const WorkList all{nullptr, nullptr, batch};
    magma_int_t rc = gemm_launch_variant<T>(v, ta, tb, g, alpha, A, B, beta, C, all, batch, max_m, max_n, s);
    return rc ? rc : launch_status();
}

// Variable size: instances bucketed by max(M, N) on the device, each bucket on its own
// auxiliary stream with its variant's tile (grid sized by the bucket's edge).
template <typename T>
static magma_int_t gemm_launch_var(magma_trans_t ta, magma_trans_t tb, const GemmSizes& g, T alpha, const T* const* A,
                                   const T* const* B, T beta, T** C, int batch, int max_m, int max_n,
                                   magma_queue_t queue) {
    const int top = gemm_bucket_of(std::max(max_m, max_n));
    int* ws = static_cast<int*>(queue_workspace(queue, sizeof(int) * bucketize_ws_ints(batch, kGemmBuckets)));
    if (!ws) return MAGMA_ERR_DEVICE_ALLOC;
    int *counts, *lists;
    int edges[kGemmBuckets];
    for (int b = 0; b < kGemmBuckets; ++b) edges[b] = std::min(kGemmEdges[b], std::max(max_m, max_n));
    magma_int_t rc = bucketize2(g.m_arr, g.n_arr, batch, edges, kGemmBuckets, queue->stream, ws, &counts, &lists);
    if (rc) return rc;
    if ((rc = queue_fork(queue))) return rc;
    const int* var = tuning().gemm_variant[sizeof(T) == 8 ? 0 : 1];
    for (int b = top; b >= 0 && !rc; --b) {
        const WorkList wl{lists + (size_t)b * batch, counts + b, 0};
        const int em = std::min(edges[b], max_m), en = std::min(edges[b], max_n);
        rc = gemm_launch_variant<T>(var[b], ta, tb, g, alpha, A, B, beta, C, wl, batch, em, en,
                                    queue_aux(queue, top - b));
    }
    queue_join(queue);
    return rc ? rc : launch_status();
}

static bool bad_trans(magma_trans_t t) { return t != MagmaNoTrans && t != MagmaTrans && t != MagmaConjTrans; }

// magmablas/dgemm_batched_core.cu:180-213: transA -1, transB -2, m -3, n -4, k -5,
// ldda -8, lddb -10, lddc -13; quick return when m, n or k <= 0.
template <typename T>
static void gemm_batched(const char* name, magma_trans_t ta, magma_trans_t tb, int m, int n, int k, T alpha,
                         const T* const* A, int lda, const T* const* B, int ldb, T beta, T** C, int ldc, int batch,
                         magma_queue_t queue) {
    int info = 0;
    if (bad_trans(ta)) info = -1;
    else if (bad_trans(tb)) info = -2;
    else if (m < 0) info = -3;
    else if (n < 0) info = -4;
    else if (k < 0) info = -5;
    else if (ta == MagmaNoTrans ? lda < m : lda < k) info = -8;
    else if (tb == MagmaNoTrans ? ldb < k : ldb < n) info = -10;
    else if (ldc < m) info = -13;
    if (info != 0) {
        magma_xerbla(name, -info);
        return;
    }
    if (m <= 0 || n <= 0 || k <= 0 || batch <= 0) return;
    GemmSizes g{m, n, k, lda, ldb, ldc, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0};
    gemm_launch<T>(ta, tb, g, alpha, A, B, beta, C, batch, m, n, queue->stream);
}

// magmablas/zgemm_vbatched.cpp:19-29 (_max_nocheck): quick return when a max is <= 0.
template <typename T>
static void gemm_vbatched_max_nocheck(magma_trans_t ta, magma_trans_t tb, int* m, int* n, int* k, T alpha,
                                      const T* const* A, int* lda, const T* const* B, int* ldb, T beta, T** C,
                                      int* ldc, int batch, int max_m, int max_n, int max_k, magma_queue_t queue) {
    if (max_m <= 0 || max_n <= 0 || max_k <= 0 || batch <= 0) return;
    GemmSizes g{0, 0, 0, 0, 0, 0, m, n, k, lda, ldb, ldc, 0};
    gemm_launch_var<T>(ta, tb, g, alpha, A, B, beta, C, batch, max_m, max_n, queue);
}

// magmablas/vbatched_check.cu:48-100 (gemm checker): transA -1, transB -2, m -3, n -4, k -5,
// ldda -8, lddb -10, lddc -13, batchCount -14. Returns the code; fills the maxima.
static int gemm_vbatched_check(magma_trans_t ta, magma_trans_t tb, int* m, int* n, int* k, int* lda, int* ldb,
                               int* ldc, int batch, magma_queue_t queue, int mx[3]) {
    if (bad_trans(ta)) return -1;
    if (bad_trans(tb)) return -2;
    if (batch < 0) return -14;
    mx[0] = mx[1] = mx[2] = 0;
    if (batch == 0) return 0;
    int r[6];
    if (reduce_sizes(m, n, k, batch, queue, r)) return MAGMA_ERR_UNKNOWN;
    if (r[3] < 0) return -3;
    if (r[4] < 0) return -4;
    if (r[5] < 0) return -5;
    int s = 0;
    if (ld_slack(ta == MagmaNoTrans ? m : k, lda, batch, queue, &s)) return MAGMA_ERR_UNKNOWN;
    if (s < 0) return -8;
    if (ld_slack(tb == MagmaNoTrans ? k : n, ldb, batch, queue, &s)) return MAGMA_ERR_UNKNOWN;
    if (s < 0) return -10;
    if (ld_slack(m, ldc, batch, queue, &s)) return MAGMA_ERR_UNKNOWN;
    if (s < 0) return -13;
    mx[0] = r[0]; mx[1] = r[1]; mx[2] = r[2];
    return 0;
}

// magmablas/vbatched_check.cu:186-262 (syrk checker): uplo -1, trans -2, n -3, k -4,
// ldda -7 (ldda < rows of A), lddc -10 (lddc < n), batchCount -11.
static int syrk_vbatched_check(magma_uplo_t uplo, magma_trans_t trans, int* n, int* k, int* lda, int* ldc,
                               int batch, magma_queue_t queue, int mx[2]) {
    if (uplo != MagmaUpper && uplo != MagmaLower) return -1;
    if (bad_trans(trans)) return -2;
    if (batch < 0) return -11;
    mx[0] = mx[1] = 0;
    if (batch == 0) return 0;
    int r[6];
    if (reduce_sizes(n, k, nullptr, batch, queue, r)) return MAGMA_ERR_UNKNOWN;
    if (r[3] < 0) return -3;
    if (r[4] < 0) return -4;
    int sl = 0;
    if (ld_slack(trans == MagmaNoTrans ? n : k, lda, batch, queue, &sl)) return MAGMA_ERR_UNKNOWN;
    if (sl < 0) return -7;
    if (ld_slack(n, ldc, batch, queue, &sl)) return MAGMA_ERR_UNKNOWN;
    if (sl < 0) return -10;
    mx[0] = r[0];
    mx[1] = r[1];
    return 0;
}

// Fixed size (magmablas/zherk_batched_core.cu:233-258): uplo -1, trans -2 (NoTrans or Trans),
// n -3, k -4, ldda < (trans == NoTrans ? n : k) -7, lddc < n -10; quick return when n or
// k is 0 (C is then left as it is, unlike the variable-size form).
template <typename T>
static void syrk_batched(const char* name, magma_uplo_t uplo, magma_trans_t trans, int n, int k, T alpha,
                         const T* const* A, int lda, T beta, T** C, int ldc, int batch, magma_queue_t queue) {
    int info = 0;
    if (uplo != MagmaUpper && uplo != MagmaLower) info = -1;
    else if (trans != MagmaNoTrans && trans != MagmaTrans) info = -2;
    else if (n < 0) info = -3;
    else if (k < 0) info = -4;
    else if (trans == MagmaNoTrans ? lda < n : lda < k) info = -7;
    else if (ldc < n) info = -10;
    if (info != 0) {
        magma_xerbla(name, -info);
        return;
    }
    if (n <= 0 || k <= 0 || batch <= 0) return;
    GemmSizes g{n, n, k, lda, lda, ldc, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                uplo == MagmaLower ? 1 : 2};
    const magma_trans_t tb = (trans == MagmaNoTrans) ? MagmaTrans : MagmaNoTrans;
    gemm_launch<T>(trans, tb, g, alpha, A, A, beta, C, batch, n, n, queue->stream);
}

// magmablas/dsyrk_vbatched_core.cu:102-112: no quick return on k (k = 0 scales the
// triangle by beta), none on n beyond an empty batch.
template <typename T>
static void syrk_vbatched_max_nocheck(magma_uplo_t uplo, magma_trans_t trans, int* n, int* k, T alpha,
                                      const T* const* A, int* lda, T beta, T** C, int* ldc, int batch, int max_n,
                                      int max_k, magma_queue_t queue) {
    (void)max_k;
    if (max_n <= 0 || batch <= 0) return;
    GemmSizes g{0, 0, 0, 0, 0, 0, n, n, k, lda, lda, ldc, uplo == MagmaLower ? 1 : 2};
    const magma_trans_t tb = (trans == MagmaNoTrans) ? MagmaTrans : MagmaNoTrans;
    gemm_launch_var<T>(trans, tb, g, alpha, A, A, beta, C, batch, max_n, max_n, queue);
}

}  // namespace mb200

using namespace mb200;

#define MB200_SYRK_FIXED_API(P, T)                                                                                    \
    void magmablas_##P##syrk_batched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t n, magma_int_t k, T alpha,  \
                                     T const* const* dA_array, magma_int_t ldda, T beta, T** dC_array,               \
                                     magma_int_t lddc, magma_int_t batchCount, magma_queue_t queue) {                \
        syrk_batched<T>(__func__, uplo, trans, n, k, alpha, dA_array, ldda, beta, dC_array, lddc, batchCount, queue); \
    }                                                                                                                 \
    void magma_##P##syrk_batched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t n, magma_int_t k, T alpha,      \
                                 T const* const* dA_array, magma_int_t ldda, T beta, T** dC_array, magma_int_t lddc, \
                                 magma_int_t batchCount, magma_queue_t queue) {                                       \
        syrk_batched<T>(__func__, uplo, trans, n, k, alpha, dA_array, ldda, beta, dC_array, lddc, batchCount, queue); \
    }

#define MB200_SYRK_API(P, T)                                                                                          \
    void magmablas_##P##syrk_vbatched_max_nocheck(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n,             \
                                                  magma_int_t* k, T alpha, T const* const* dA_array,                  \
                                                  magma_int_t* ldda, T beta, T** dC_array, magma_int_t* lddc,         \
                                                  magma_int_t batchCount, magma_int_t max_n, magma_int_t max_k,       \
                                                  magma_queue_t queue) {                                              \
        syrk_vbatched_max_nocheck<T>(uplo, trans, n, k, alpha, dA_array, ldda, beta, dC_array, lddc, batchCount,     \
                                     max_n, max_k, queue);                                                            \
    }                                                                                                                 \
    void magmablas_##P##syrk_vbatched_max(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,     \
                                          T alpha, T const* const* dA_array, magma_int_t* ldda, T beta,               \
                                          T** dC_array, magma_int_t* lddc, magma_int_t batchCount, magma_int_t max_n, \
                                          magma_int_t max_k, magma_queue_t queue) {                                   \
        int mx[2];                                                                                                    \
        const int info = syrk_vbatched_check(uplo, trans, n, k, ldda, lddc, batchCount, queue, mx);                  \
        if (info != 0) {                                                                                              \
            magma_xerbla(__func__, -info);                                                                            \
            return;                                                                                                   \
        }                                                                                                             \
        syrk_vbatched_max_nocheck<T>(uplo, trans, n, k, alpha, dA_array, ldda, beta, dC_array, lddc, batchCount,     \
                                     max_n, max_k, queue);                                                            \
    }                                                                                                                 \
    void magmablas_##P##syrk_vbatched_nocheck(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k, \
                                              T alpha, T const* const* dA_array, magma_int_t* ldda, T beta,           \
                                              T** dC_array, magma_int_t* lddc, magma_int_t batchCount,                \
                                              magma_queue_t queue) {                                                  \
        int r[6];                                                                                                     \
        if (batchCount <= 0 || reduce_sizes(n, k, nullptr, batchCount, queue, r)) return;                            \
        syrk_vbatched_max_nocheck<T>(uplo, trans, n, k, alpha, dA_array, ldda, beta, dC_array, lddc, batchCount,     \
                                     r[0], r[1], queue);                                                              \
    }                                                                                                                 \
    void magmablas_##P##syrk_vbatched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,         \
                                      T alpha, T const* const* dA_array, magma_int_t* ldda, T beta, T** dC_array,     \
                                      magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue) {               \
        int mx[2];                                                                                                    \
        const int info = syrk_vbatched_check(uplo, trans, n, k, ldda, lddc, batchCount, queue, mx);                  \
        if (info != 0) {                                                                                              \
            magma_xerbla(__func__, -info);                                                                            \
            return;                                                                                                   \
        }                                                                                                             \
        syrk_vbatched_max_nocheck<T>(uplo, trans, n, k, alpha, dA_array, ldda, beta, dC_array, lddc, batchCount,     \
                                     mx[0], mx[1], queue);                                                            \
    }

#define MB200_GEMM_API(P, T)                                                                                          \
    void magmablas_##P##gemm_batched(magma_trans_t ta, magma_trans_t tb, magma_int_t m, magma_int_t n, magma_int_t k, \
                                     T alpha, T const* const* dA_array, magma_int_t ldda, T const* const* dB_array,   \
                                     magma_int_t lddb, T beta, T** dC_array, magma_int_t lddc, magma_int_t batchCount, \
                                     magma_queue_t queue) {                                                           \
        gemm_batched<T>(__func__, ta, tb, m, n, k, alpha, dA_array, ldda, dB_array, lddb, beta, dC_array, lddc,       \
                        batchCount, queue);                                                                           \
    }                                                                                                                 \
    void magma_##P##gemm_batched(magma_trans_t ta, magma_trans_t tb, magma_int_t m, magma_int_t n, magma_int_t k,     \
                                 T alpha, T const* const* dA_array, magma_int_t ldda, T const* const* dB_array,       \
                                 magma_int_t lddb, T beta, T** dC_array, magma_int_t lddc, magma_int_t batchCount,     \
                                 magma_queue_t queue) {                                                               \
        gemm_batched<T>(__func__, ta, tb, m, n, k, alpha, dA_array, ldda, dB_array, lddb, beta, dC_array, lddc,       \
                        batchCount, queue);                                                                           \
    }                                                                                                                 \
    void magmablas_##P##gemm_vbatched_max_nocheck(                                                                    \
        magma_trans_t ta, magma_trans_t tb, magma_int_t* m, magma_int_t* n, magma_int_t* k, T alpha,                  \
        T const* const* dA_array, magma_int_t* ldda, T const* const* dB_array, magma_int_t* lddb, T beta,             \
        T** dC_array, magma_int_t* lddc, magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,                \
        magma_int_t max_k, magma_queue_t queue) {                                                                     \
        gemm_vbatched_max_nocheck<T>(ta, tb, m, n, k, alpha, dA_array, ldda, dB_array, lddb, beta, dC_array, lddc,    \
                                     batchCount, max_m, max_n, max_k, queue);                                        \
    }                                                                                                                 \
    void magmablas_##P##gemm_vbatched_max(magma_trans_t ta, magma_trans_t tb, magma_int_t* m, magma_int_t* n,         \
                                          magma_int_t* k, T alpha, T const* const* dA_array, magma_int_t* ldda,       \
                                          T const* const* dB_array, magma_int_t* lddb, T beta, T** dC_array,          \
                                          magma_int_t* lddc, magma_int_t batchCount, magma_int_t max_m,               \
                                          magma_int_t max_n, magma_int_t max_k, magma_queue_t queue) {                \
        int mx[3];                                                                                                    \
        const int info = gemm_vbatched_check(ta, tb, m, n, k, ldda, lddb, lddc, batchCount, queue, mx);              \
        if (info != 0) {                                                                                              \
            magma_xerbla(__func__, -info);                                                                            \
            return;                                                                                                   \
        }                                                                                                             \
        gemm_vbatched_max_nocheck<T>(ta, tb, m, n, k, alpha, dA_array, ldda, dB_array, lddb, beta, dC_array, lddc,    \
                                     batchCount, max_m, max_n, max_k, queue);                                        \
    }                                                                                                                 \
    void magmablas_##P##gemm_vbatched_nocheck(magma_trans_t ta, magma_trans_t tb, magma_int_t* m, magma_int_t* n,     \
                                              magma_int_t* k, T alpha, T const* const* dA_array, magma_int_t* ldda,   \
                                              T const* const* dB_array, magma_int_t* lddb, T beta, T** dC_array,      \
                                              magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue) {       \
        int r[6];                                                                                                     \
        if (batchCount <= 0 || reduce_sizes(m, n, k, batchCount, queue, r)) return;                                   \
        gemm_vbatched_max_nocheck<T>(ta, tb, m, n, k, alpha, dA_array, ldda, dB_array, lddb, beta, dC_array, lddc,    \
                                     batchCount, r[0], r[1], r[2], queue);                                            \
    }                                                                                                                 \
    void magmablas_##P##gemm_vbatched(magma_trans_t ta, magma_trans_t tb, magma_int_t* m, magma_int_t* n,             \
                                      magma_int_t* k, T alpha, T const* const* dA_array, magma_int_t* ldda,           \
                                      T const* const* dB_array, magma_int_t* lddb, T beta, T** dC_array,              \
                                      magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue) {               \
        int mx[3];                                                                                                    \
        const int info = gemm_vbatched_check(ta, tb, m, n, k, ldda, lddb, lddc, batchCount, queue, mx);              \
        if (info != 0) {                                                                                              \
            magma_xerbla(__func__, -info);                                                                            \
            return;                                                                                                   \
        }                                                                                                             \
        gemm_vbatched_max_nocheck<T>(ta, tb, m, n, k, alpha, dA_array, ldda, dB_array, lddb, beta, dC_array, lddc,    \
                                     batchCount, mx[0], mx[1], mx[2], queue);                                        \
    }

extern "C" {
MB200_GEMM_API(d, double)
MB200_GEMM_API(s, float)
MB200_SYRK_API(d, double)
MB200_SYRK_API(s, float)
MB200_SYRK_FIXED_API(d, double)
MB200_SYRK_FIXED_API(s, float)
}
