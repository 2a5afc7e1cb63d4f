// lu_tc.cu -- FP32-accurate batched LU with the trailing matrix resident in
// tensor memory and its updates on the tensor cores (tcgen05, kind::tf32).
//
// Used by the mixed-precision solve (magma_dsgesv_batched) for n <= 256, n a
// multiple of 32, in place of conversion + FP32 CUDA-core LU. One CTA per SM
// walks the batch; per instance:
//   1. thread t reads row t of the FP64 matrix once, converts it to FP32 into
//      TMEM (rows 0..127: lanes 0..127, columns 0..255; rows 128..255: the same
//      lanes, columns 256..511 -- the whole 256 KB of TMEM holds the matrix),
//      and forms ||A||_inf and the overflow test on the way (dlag2s + dlange);
//   2. for each 32-column panel: the panel is read from TMEM into registers and
//      factored with the register pivot steps of small_lu.cuh (rows never move;
//      each thread tracks its row's LAPACK position); a row chosen as a pivot
//      is final and is stored to the output at its position; the pivot rows'
//      trailing entries are gathered to shared memory and solved with L11
//      (U12), and the trailing update A22 -= L21 U12 runs on the tensor cores
//      as three TF32 products per K step (lo*hi + hi*lo + hi*hi of the split
//      operands, accumulating in FP32 in TMEM), which carries ~21 bits of each
//      product -- single-precision quality, enough for FP64 refinement to
//      converge for kappa up to ~1e6 as with a CUDA-core FP32 LU.
// The CUDA cores do the pivoting while the tensor cores do ~80% of the flops;
// the FP64 matrix is read from HBM once and the factors written once.
// Every wait on the tensor core is bounded: on time-out the kernel raises an
// error flag, frees its TMEM and returns.
#include "internal.h"
#include "small_lu.cuh"
#include "tc_ptx.cuh"
#include "lu_tc.h"
#include <cfloat>
#include <cstddef>
#include <atomic>
#include <climits>

namespace mb200 {

constexpr int kTcNT = 256;        // threads = matrix rows (n <= 256)
constexpr int kTcTrail = 224;     // trailing columns of the first panel at n = 256

// Panel factorisation of the FP32 LU (8 warps, thread t = row t, 32 columns in
// registers). The pivot choice need not match LAPACK's bit for bit here (the FP64
// refinement and its fallback own the accuracy), which allows a cheaper step than
// the FP64 kernels' exact one:
//  * packed keys: |a(i,k)|'s bit pattern without its low 8 mantissa bits, plus one,
//    shifted back up, with 255 - row in the low byte, so one unsigned max reduction
//    picks the largest magnitude (to 15 mantissa bits: a pivot within a factor
//    1 + 2^-15 of the column maximum) and names its row; no ballot or position
//    reduction follows, and every candidate's key is above a non-candidate's 0;
//  * one barrier per step: before it, each warp's best row publishes its key,
//    position, approximate reciprocal and columns into its warp's slot (slots
//    double-buffered by step parity); after it, every warp reduces the 8 slot keys
//    and reads the winner's row;
//  * the multiplier is a(i,k) * (1/pivot) with the reciprocal to ~2 ulp.
struct TcPanelShared {
    alignas(16) float cand[2][kTcNT / 32][32];
    float cinv[2][kTcNT / 32];
    int cpos[2][kTcNT / 32];
    unsigned ckey[2][kTcNT / 32];
};

__device__ __forceinline__ void tc_panel_steps(float (&a)[32], int n, int k0, int t, int& pos, int& my_ipiv,
                                               int& info, TcPanelShared& sh) {
    const int lane = t & 31, w = t >> 5;
    static_for<0, 32>([&](auto kc) {
        constexpr int k = decltype(kc)::value;
        constexpr int buf = k & 1;
        constexpr int jw = k & ~3;
        const int g = k0 + k;
        const bool cand = (pos >= g) && (t < n);
        // candidates: ((|x| bits >> 8) + 1) << 8 | (255 - row) >= 0x100 > 0 = not a candidate
        const unsigned key = cand ? ((((__float_as_uint(fabsf(a[k])) >> 8) + 1u) << 8) | (255u - unsigned(t))) : 0u;
        const unsigned wmax = __reduce_max_sync(kFullMask, key);
        if (lane == 0) sh.ckey[buf][w] = wmax;
        if (wmax != 0u && key == wmax) {   // this warp's best row (unique: the key names it)
            sh.cpos[buf][w] = pos;
            sh.cinv[buf][w] = __fdividef(1.0f, a[k]);
            float4* dst = reinterpret_cast<float4*>(&sh.cand[buf][w][0]);
#pragma unroll
            for (int j = jw; j < 32; j += 4) dst[j / 4] = make_float4(a[j], a[j + 1], a[j + 2], a[j + 3]);
        }
        __syncthreads();
        const unsigned gmax = __reduce_max_sync(kFullMask, lane < kTcNT / 32 ? sh.ckey[buf][lane] : 0u);
        const int s = 255 - int(gmax & 0xFFu);   // the pivot row's thread
        const int ws = (s >> 5) & (kTcNT / 32 - 1);
        const float* prow = &sh.cand[buf][ws][0];
        const float piv = prow[k];
        const int p = sh.cpos[buf][ws];
        if (t == g) my_ipiv = (piv != 0.0f) ? p + 1 : g + 1;   // a zero pivot interchanges nothing
        if (piv != 0.0f) {
            if (pos == g) pos = p;   // the row at position g takes the pivot's old position
            if (t == s) pos = g;
        } else if (info == 0) {
            info = g + 1;
        }
        if (pos > g && t < n) {
            if (piv != 0.0f) a[k] = a[k] * sh.cinv[buf][ws];
            const float l = a[k];
            const float4* r4 = reinterpret_cast<const float4*>(prow);
#pragma unroll
            for (int j = jw; j < 32; j += 4) {
                const float4 u = r4[j / 4];
                if (j > k) a[j] = fmaf(l, -u.x, a[j]);
                if (j + 1 > k) a[j + 1] = fmaf(l, -u.y, a[j + 1]);
                if (j + 2 > k) a[j + 2] = fmaf(l, -u.z, a[j + 2]);
                if (j + 3 > k) a[j + 3] = fmaf(l, -u.w, a[j + 3]);
            }
        }
    });
}

struct TcLuSmem {
    // The L21 operand is built after the pivot rows' entries (Ug) have been solved and
    // copied into the B operand, and the MMA that reads it completes before the next
    // panel gathers into Ug, so the two share storage.
    union {
        float A[2][2][128 * 32];    // L21 operand: [row half][hi, lo], K-major canonical (16 KB each)
        float Ug[32][kTcTrail + 1]; // pivot rows' trailing entries; U12 after the solve
    };
    float B[2][kTcTrail * 32];      // U12 operand: [hi, lo], K-major canonical (28 KB each)
    // each panel's 32x32 diagonal block by position: L11 below the diagonal, U11 on
    // and above it (the trsm reads the current one; the refinement inverts them all)
    float dblk[kTcNT / 32][32][33];
    TcPanelShared pan;
    double red[kTcNT / 32];
    unsigned long long mbar;
    uint32_t tmem_base;
};

// Float index of (row, k) in a K-major no-swizzle operand: 8x4 core matrices of
// 128 bytes; K-adjacent core matrices 128 bytes apart (LBO), row groups 1024 (SBO).
__device__ __forceinline__ int kmajor(int row, int k) {
    return (((row >> 3) * 8 + (k >> 2)) * 8 + (row & 7)) * 4 + (k & 3);
}
constexpr uint32_t kLbo = 128, kSbo = 1024;

// U12 = L11^-1 A12 for column c of sh.Ug (unit lower L11), rows in groups of 8.
__device__ __forceinline__ void tc_trsm_column(TcLuSmem& sh, const float (&L11)[32][33], int c) {
#pragma unroll 1
    for (int q0 = 0; q0 < 32; q0 += 8) {
        float x[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) x[r] = sh.Ug[q0 + r][c];
        for (int rr = 0; rr < q0; ++rr) {
            const float u = sh.Ug[rr][c];
#pragma unroll
            for (int r = 0; r < 8; ++r) x[r] = fmaf(L11[q0 + r][rr], -u, x[r]);
        }
        static_for<0, 8>([&](auto rc) {
            constexpr int rr = decltype(rc)::value;
#pragma unroll
            for (int r = rr + 1; r < 8; ++r) x[r] = fmaf(L11[q0 + r][q0 + rr], -x[rr], x[r]);
        });
#pragma unroll
        for (int r = 0; r < 8; ++r) sh.Ug[q0 + r][c] = x[r];
    }
}

// L2 retention policy and loads that carry it (PTX createpolicy / ld .L2::cache_hint).
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ double ld_keep(const double* p, uint64_t pol) {
    double v;
    asm("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double2 ld_keep2(const double* p, uint64_t pol) {   // p 16-byte aligned
    double2 v;
    asm("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
    return v;
}

// ---------------------------------------------------------------------------
// Refinement in the block that factored the instance (magma_dsgesv_gpu's loop,
// src/zcgesv_gpu.cpp:251-362: ITERMAX 30, BWDMAX 1). The single-precision solves
// read L from tensor memory (each row's own TMEM lane holds its multipliers), U12
// from the rows stored in global memory during the factorisation (L2-resident),
// and the inverses of the 32x32 diagonal blocks formed here from the panels'
// diagonal blocks; the FP64 residual reads A again (kept in L2 at a high retention
// priority since the conversion read it). Thread t owns row t of A, B and the residual, and the
// solution entry of column pos (the position its row took).
constexpr int kTcR = 4;          // right-hand sides per refinement pass (the residual reads them as a double4)
constexpr int kTcItermax = 30;

struct TcRefineSmem {            // overlays the operand buffers once the factorisation is done
    float inv[kTcNT / 32][2][32][33];   // [block][0: L^-1 (unit lower), 1: U^-1][row][col]
    float f[kTcNT][kTcR];               // single-precision vectors by position
    alignas(32) double xs[kTcNT][kTcR]; // FP64 solution by column, for the residual
    double red[2][kTcNT / 32][kTcR];
    alignas(32) double part[2][kTcNT][kTcR];   // the residual's two column halves, per row
};

// L^-1 (unit lower part) and U^-1 (upper part) of one diagonal block, one warp:
// lane j forms column j of each by substitution on e_j.
__device__ __forceinline__ void tc_invert_block(const float (&blk)[32][33], float (&linv)[32][33],
                                                float (&uinv)[32][33], int lane) {
    float x[32];
    static_for<0, 32>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        float s = (i == lane) ? 1.0f : 0.0f;
#pragma unroll
        for (int k = 0; k < i; ++k) s = fmaf(-blk[i][k], x[k], s);
        x[i] = (i < lane) ? 0.0f : s;
    });
#pragma unroll
    for (int i = 0; i < 32; ++i) linv[i][lane] = x[i];
    static_for<0, 32>([&](auto ic) {
        constexpr int i = 31 - decltype(ic)::value;
        float s = (i == lane) ? 1.0f : 0.0f;
#pragma unroll
        for (int k = i + 1; k < 32; ++k) s = fmaf(-blk[i][k], x[k], s);
        x[i] = (i > lane) ? 0.0f : s / blk[i][i];
    });
#pragma unroll
    for (int i = 0; i < 32; ++i) uinv[i][lane] = x[i];
}

// c_J = inv * f_J for the 32 positions of block J, by warp J (lane i: row i).
// Four partial sums per entry keep the dependent fma chains 8 long.
__device__ __forceinline__ void tc_block_diag(const float (&inv)[32][33], float (&f)[kTcNT][kTcR], int j0, int lane) {
    float c[4][kTcR];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < kTcR; ++r) c[q][r] = 0.0f;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        const float l = inv[lane][k];
        const float4 fk = *reinterpret_cast<const float4*>(&f[j0 + k][0]);
        c[k & 3][0] = fmaf(l, fk.x, c[k & 3][0]);
        c[k & 3][1] = fmaf(l, fk.y, c[k & 3][1]);
        c[k & 3][2] = fmaf(l, fk.z, c[k & 3][2]);
        c[k & 3][3] = fmaf(l, fk.w, c[k & 3][3]);
    }
    __syncwarp();   // every lane has read f_J before it is overwritten
#pragma unroll
    for (int r = 0; r < kTcR; ++r) f[j0 + lane][r] = (c[0][r] + c[1][r]) + (c[2][r] + c[3][r]);
}

// fo -= sum_k v[k] * f[j0 + k], with four partial sums (chains 8 long).
__device__ __forceinline__ void tc_block_update(float (&fo)[kTcR], const float (&v)[32],
                                                const float (&f)[kTcNT][kTcR], int j0) {
    float d[4][kTcR];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < kTcR; ++r) d[q][r] = 0.0f;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        const float4 fk = *reinterpret_cast<const float4*>(&f[j0 + k][0]);
        d[k & 3][0] = fmaf(v[k], fk.x, d[k & 3][0]);
        d[k & 3][1] = fmaf(v[k], fk.y, d[k & 3][1]);
        d[k & 3][2] = fmaf(v[k], fk.z, d[k & 3][2]);
        d[k & 3][3] = fmaf(v[k], fk.w, d[k & 3][3]);
    }
#pragma unroll
    for (int r = 0; r < kTcR; ++r) fo[r] -= (d[0][r] + d[1][r]) + (d[2][r] + d[3][r]);
}

// L U c = f in single precision, f by position in rf.f (written by the caller);
// on return fo holds c at this thread's position. One barrier pair per 32-row block.
__device__ __forceinline__ void tc_solve(float (&fo)[kTcR], int pos, bool live, int lane, int w, int nb,
                                         uint32_t trow, const float* __restrict__ S, int n, TcRefineSmem& rf) {
    // forward: unit lower L, blocks ascending; rows below the block take its update
    for (int J = 0; J < nb; ++J) {
        const int j0 = J << 5;
        float lv[32];
        tc::tmem_ld32(trow + j0, lv);   // this row's columns j0..j0+31 (L entries when pos >= j0 + 32)
        if (w == J) tc_block_diag(rf.inv[J][0], rf.f, j0, lane);
        tc::wait_ld();
        __syncthreads();
        if (J + 1 < nb) {
            if (live && pos >= j0 + 32) {
                tc_block_update(fo, lv, rf.f, j0);
#pragma unroll
                for (int r = 0; r < kTcR; ++r) rf.f[pos][r] = fo[r];
            }
            __syncthreads();
        }
    }
    if (live) {
#pragma unroll
        for (int r = 0; r < kTcR; ++r) fo[r] = rf.f[pos][r];
    }
    // backward: U, blocks descending; rows above the block take its update. A row's
    // U entries of block J are 32 contiguous floats of its row-major U12 row; the next
    // block's are loaded while this block's step runs.
    float uv[32], un[32];
    auto load_u = [&](int J, float (&dst)[32]) {
        if (live && pos < (J << 5)) {
            const float4* src = reinterpret_cast<const float4*>(S + (size_t)pos * n + (J << 5));
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 v = src[q];
                dst[4 * q] = v.x; dst[4 * q + 1] = v.y; dst[4 * q + 2] = v.z; dst[4 * q + 3] = v.w;
            }
        }
    };
    load_u(nb - 1, uv);
    for (int J = nb - 1; J >= 0; --J) {
        const int j0 = J << 5;
        const bool above = live && pos < j0;
        if (J > 0) load_u(J - 1, un);
        if (w == J) tc_block_diag(rf.inv[J][1], rf.f, j0, lane);
        __syncthreads();
        if (J > 0) {
            if (above) {
                tc_block_update(fo, uv, rf.f, j0);
#pragma unroll
                for (int r = 0; r < kTcR; ++r) rf.f[pos][r] = fo[r];
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < 32; ++k) uv[k] = un[k];
        }
    }
    if (live) {
#pragma unroll
        for (int r = 0; r < kTcR; ++r) fo[r] = rf.f[pos][r];
    }
}

// Block-wide maxima of v and u per right-hand side (every thread gets them).
__device__ __forceinline__ void tc_max2(double (&v)[kTcR], double (&u)[kTcR], int lane, int w, TcRefineSmem& rf) {
#pragma unroll
    for (int r = 0; r < kTcR; ++r) {
        for (int off = 16; off > 0; off >>= 1) {
            v[r] = fmax(v[r], __shfl_xor_sync(kFullMask, v[r], off));
            u[r] = fmax(u[r], __shfl_xor_sync(kFullMask, u[r], off));
        }
    }
    __syncthreads();   // the previous maxima have been read
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < kTcR; ++r) {
            rf.red[0][w][r] = v[r];
            rf.red[1][w][r] = u[r];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kTcR; ++r) {
        v[r] = 0.0;
        u[r] = 0.0;
        for (int k = 0; k < kTcNT / 32; ++k) {
            v[r] = fmax(v[r], rf.red[0][k][r]);
            u[r] = fmax(u[r], rf.red[1][k][r]);
        }
    }
}

// Returns iter: >= 0 refinement passes after the first solve, -2 when a residual does
// not fit single precision, -31 when it does not converge (or stalls: the ratio of
// residual to its bound fails to halve twice in a row).
__device__ int tc_refine_instance(const TcLuArgs& g, int id, int t, int lane, int w, int pos, uint32_t trow,
                                  const float* __restrict__ S, TcRefineSmem& rf, uint64_t keep) {
    const int n = g.n, nb = n >> 5;
    const bool live = t < n;
    const double* A = g.dA[id];
    const double* Bv = g.dB[id];
    double* X = g.dX[id];
    const double cte = g.anrm[id] * (DBL_EPSILON * 0.5) * sqrt((double)n);
    // residual by row pairs when every row pair is 16-byte aligned (even lda, aligned A)
    const bool pairs = (g.lda % 2 == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
    int iter_out = 0;
    for (int c0 = 0; c0 < g.nrhs && iter_out >= 0; c0 += kTcR) {
        double b[kTcR], x[kTcR], res[kTcR];
#pragma unroll
        for (int r = 0; r < kTcR; ++r) {
            b[r] = (live && c0 + r < g.nrhs) ? Bv[t + (size_t)(c0 + r) * g.ldb] : 0.0;
            x[r] = 0.0;
            res[r] = b[r];
        }
        int iiter = 0, stalls = 0;
        double prev_ratio = 1e300;
        for (;;) {
            bool ovf = false;
            float fo[kTcR];
#pragma unroll
            for (int r = 0; r < kTcR; ++r) {
                ovf |= !(fabs(res[r]) <= (double)FLT_MAX);
                fo[r] = (float)res[r];
            }
            if (__syncthreads_or(ovf)) { iter_out = -2; break; }
            if (live) {
#pragma unroll
                for (int r = 0; r < kTcR; ++r) rf.f[pos][r] = fo[r];   // P r
            }
            __syncthreads();
            tc_solve(fo, pos, live, lane, w, nb, trow, S, n, rf);
            if (live) {
#pragma unroll
                for (int r = 0; r < kTcR; ++r) {
                    x[r] += (double)fo[r];
                    rf.xs[pos][r] = x[r];
                }
            }
            __syncthreads();
            // R = B - A X in double precision
#pragma unroll
            for (int r = 0; r < kTcR; ++r) res[r] = b[r];
            if (pairs) {
                // thread t: rows 2(t%128) and 2(t%128)+1 over column half t/128, 16-byte
                // loads (two rows per load), 16 columns in flight; halves summed per row
                const int rp = 2 * (t & 127), h = t >> 7, jh = n >> 1;
                double p0[kTcR], p1[kTcR];
#pragma unroll
                for (int r = 0; r < kTcR; ++r) p0[r] = p1[r] = 0.0;
                for (int j0 = h * jh; rp < n && j0 < (h + 1) * jh; j0 += 16) {
                    double2 av[16];
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) av[jj] = ld_keep2(A + rp + (size_t)(j0 + jj) * g.lda, keep);
#pragma unroll
                    for (int jj = 0; jj < 16; ++jj) {
                        const double4 xj = *reinterpret_cast<const double4*>(&rf.xs[j0 + jj][0]);
                        p0[0] = fma(av[jj].x, xj.x, p0[0]); p1[0] = fma(av[jj].y, xj.x, p1[0]);
                        p0[1] = fma(av[jj].x, xj.y, p0[1]); p1[1] = fma(av[jj].y, xj.y, p1[1]);
                        p0[2] = fma(av[jj].x, xj.z, p0[2]); p1[2] = fma(av[jj].y, xj.z, p1[2]);
                        p0[3] = fma(av[jj].x, xj.w, p0[3]); p1[3] = fma(av[jj].y, xj.w, p1[3]);
                    }
                }
                if (rp < n) {
                    *reinterpret_cast<double4*>(&rf.part[h][rp][0]) = make_double4(p0[0], p0[1], p0[2], p0[3]);
                    *reinterpret_cast<double4*>(&rf.part[h][rp + 1][0]) = make_double4(p1[0], p1[1], p1[2], p1[3]);
                }
                __syncthreads();
                if (live) {
#pragma unroll
                    for (int r = 0; r < kTcR; ++r) res[r] = b[r] - (rf.part[0][t][r] + rf.part[1][t][r]);
                }
            } else if (live) {
                // 32 columns at a time: all 32 loads in flight before their fma's
                for (int j0 = 0; j0 < n; j0 += 32) {
                    double av[32];
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) av[jj] = ld_keep(A + t + (size_t)(j0 + jj) * g.lda, keep);
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) {
                        const double4 xj = *reinterpret_cast<const double4*>(&rf.xs[j0 + jj][0]);
                        res[0] = fma(-av[jj], xj.x, res[0]);
                        res[1] = fma(-av[jj], xj.y, res[1]);
                        res[2] = fma(-av[jj], xj.z, res[2]);
                        res[3] = fma(-av[jj], xj.w, res[3]);
                    }
                }
            }
            double xn[kTcR], rn[kTcR];
#pragma unroll
            for (int r = 0; r < kTcR; ++r) {
                const bool v = live && c0 + r < g.nrhs;
                xn[r] = v ? fabs(x[r]) : 0.0;
                rn[r] = v ? fabs(res[r]) : 0.0;
            }
            tc_max2(xn, rn, lane, w, rf);
            bool ok = true;
            double ratio = 0.0;
#pragma unroll
            for (int r = 0; r < kTcR; ++r) {
                if (c0 + r < g.nrhs) {
                    ok &= (rn[r] <= xn[r] * cte);
                    ratio = fmax(ratio, rn[r] / fmax(xn[r] * cte, DBL_MIN));
                }
            }
            if (ok) break;
            ++iiter;
            stalls = (ratio > 0.5 * prev_ratio) ? stalls + 1 : 0;
            prev_ratio = ratio;
            if (iiter >= kTcItermax || stalls >= 2) { iter_out = -kTcItermax - 1; break; }
        }
        if (iter_out < 0) break;
        iter_out = max(iter_out, iiter);
        if (live) {
#pragma unroll
            for (int r = 0; r < kTcR; ++r)
                if (c0 + r < g.nrhs) X[pos + (size_t)(c0 + r) * g.ldx] = x[r];
        }
        __syncthreads();
    }
    return iter_out;
}

__global__ void __launch_bounds__(kTcNT, 1)
lu_tf32x3_kernel(TcLuArgs g) {
    extern __shared__ unsigned char tc_smem_raw[];
    // 1024-byte alignment of the operand buffers (descriptors address 16-byte units)
    const uint32_t raw = tc::smem_addr(tc_smem_raw);
    TcLuSmem& sh = *reinterpret_cast<TcLuSmem*>(tc_smem_raw + (((raw + 1023u) & ~1023u) - raw));
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, half = t >> 7;
    const int n = g.n;
    const uint32_t mbar = tc::smem_addr(&sh.mbar);
    if (w == 0) {
        tc::tmem_alloc(tc::smem_addr(&sh.tmem_base), 512);
        tc::tmem_relinquish();
    }
    if (t == 0) {
        tc::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = sh.tmem_base;
    // this thread's lane (row t): lane field 32*(w%4) + lane (implicit), column base half*256
    const uint32_t trow = tbase + (uint32_t(32 * (w & 3)) << 16) + uint32_t(half * 256);
    uint32_t phase = 0;
    bool failed = false;
    const uint64_t keep = l2_evict_last_policy();
    for (int id = blockIdx.x; id < g.batch && !failed; id += gridDim.x) {
        const double* A = g.dA[id];
        float* S = g.SA + (size_t)id * n * n;
        // ---- 1. FP64 row -> FP32 TMEM, row sums, overflow ----
        // A is read with a high L2 retention priority: the refinement passes read it
        // again, and the instances in flight (one per SM, 512 KB each at n = 256) fit L2
        double rs = 0.0;
        bool ovf = false;
        for (int c0 = 0; c0 < n; c0 += 32) {
            float v[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const double a = (t < n) ? ld_keep(A + t + (size_t)(c0 + c) * g.lda, keep) : 0.0;
                rs += fabs(a);
                ovf |= !(fabs(a) <= (double)FLT_MAX);
                v[c] = (float)a;
            }
            tc::tmem_st32(trow + c0, v);
        }
        tc::wait_st();
        for (int off = 16; off > 0; off >>= 1) rs = fmax(rs, __shfl_xor_sync(kFullMask, rs, off));
        if (lane == 0) sh.red[w] = rs;
        tc::fence_before_sync();
        const int any_ovf = __syncthreads_or(ovf);
        tc::fence_after_sync();
        if (t == 0) {
            double m = 0.0;
            for (int k = 0; k < kTcNT / 32; ++k) m = fmax(m, sh.red[k]);
            g.anrm[id] = m;
            g.iter[id] = any_ovf ? -2 : 0;
            if (any_ovf) g.fail_list[atomicAdd(g.fail_count, 1)] = id;
        }
        if (any_ovf) {          // block-uniform: the FP64 fallback takes this instance
            __syncthreads();
            continue;
        }
        // ---- 2. panels ----
        int pos = (t < n) ? t : INT_MAX / 2;
        int info = 0;
        for (int k0 = 0; k0 < n && !failed; k0 += 32) {
            float a[32];
            tc::tmem_ld32(trow + k0, a);
            tc::wait_ld();
            int my_ipiv = 0;
            tc_panel_steps(a, n, k0, t, pos, my_ipiv, info, sh.pan);
            if (t >= k0 && t < k0 + 32) g.ipiv[id][t] = my_ipiv;
            const bool piv = (t < n) && pos >= k0 && pos < k0 + 32;
            const int ncols = n - k0 - 32;
            tc::tmem_st32(trow + k0, a);   // this row's panel entries, kept until it is stored
            if (piv) {
#pragma unroll
                for (int c = 0; c < 32; ++c) sh.dblk[k0 >> 5][pos - k0][c] = a[c];
            }
            // a pivot row is final: the panel from registers now, its trailing entries to
            // shared memory for the U12 solve, and its columns left of the panel (which
            // stay untouched in TMEM) once the whole factorisation is done
            if (__any_sync(kFullMask, piv)) {
                for (int c0 = k0 + 32; c0 < n; c0 += 32) {
                    float v[32];
                    tc::tmem_ld32(trow + c0, v);
                    tc::wait_ld();
                    if (piv) {
#pragma unroll
                        for (int c = 0; c < 32; ++c) sh.Ug[pos - k0][c0 - k0 - 32 + c] = v[c];
                    }
                }
            }
            tc::wait_st();
            __syncthreads();
            if (ncols <= 0) break;
            for (int c = t; c < ncols; c += kTcNT) tc_trsm_column(sh, sh.dblk[k0 >> 5], c);
            __syncthreads();
            // U12 rows to global memory (read by the refinement's backward sweeps), and the
            // split B operand
            // (row-major: position k0 + r, columns k0 + 32 ..; one row is contiguous)
            for (int idx = t; idx < 32 * ncols; idx += kTcNT) {
                const int c = idx % ncols, r = idx / ncols;
                S[(size_t)(k0 + r) * n + (k0 + 32 + c)] = sh.Ug[r][c];
            }
            for (int f = t; f < 32 * ncols; f += kTcNT) {
                const int k = (f & 3) | (((f >> 5) & 7) << 2);
                const int c = ((f >> 2) & 7) | ((f >> 8) << 3);
                float hi, lo;
                tc::split_tf32(sh.Ug[k][c], hi, lo);
                sh.B[0][f] = hi;
                sh.B[1][f] = lo;
            }
            __syncthreads();   // Ug fully read before the A operand overwrites it
            // A operand: this row's multipliers (zero for rows already placed)
            {
                const bool live = (t < n) && pos >= k0 + 32;
                const int r = t & 127;
#pragma unroll
                for (int kq = 0; kq < 8; ++kq) {
                    float4 h4, l4;
                    tc::split_tf32(live ? a[4 * kq + 0] : 0.0f, h4.x, l4.x);
                    tc::split_tf32(live ? a[4 * kq + 1] : 0.0f, h4.y, l4.y);
                    tc::split_tf32(live ? a[4 * kq + 2] : 0.0f, h4.z, l4.z);
                    tc::split_tf32(live ? a[4 * kq + 3] : 0.0f, h4.w, l4.w);
                    *reinterpret_cast<float4*>(&sh.A[half][0][kmajor(r, 4 * kq)]) = h4;
                    *reinterpret_cast<float4*>(&sh.A[half][1][kmajor(r, 4 * kq)]) = l4;
                }
            }
            tc::fence_proxy_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            if (t == 0 && g.issue_mma) {
                tc::fence_after_sync();
                const uint32_t idesc = tc::idesc_tf32(128, ncols, true);   // D += (-L21) U12
                const int halves = (n + 127) / 128;
                for (int h = 0; h < halves; ++h) {
                    const uint32_t d = tbase + uint32_t(h * 256 + k0 + 32);
#pragma unroll
                    for (int s = 0; s < 4; ++s) {   // K = 32 in steps of 8 (two core matrices)
                        const uint64_t ah = tc::smem_desc(tc::smem_addr(&sh.A[h][0][s * 64]), kLbo, kSbo);
                        const uint64_t al = tc::smem_desc(tc::smem_addr(&sh.A[h][1][s * 64]), kLbo, kSbo);
                        const uint64_t bh = tc::smem_desc(tc::smem_addr(&sh.B[0][s * 64]), kLbo, kSbo);
                        const uint64_t bl = tc::smem_desc(tc::smem_addr(&sh.B[1][s * 64]), kLbo, kSbo);
                        tc::mma_tf32(d, al, bh, idesc, true);
                        tc::mma_tf32(d, ah, bl, idesc, true);
                        tc::mma_tf32(d, ah, bh, idesc, true);
                    }
                }
                tc::commit(mbar);
            }
            // bounded wait for the update (about 4 s unless the test hook shortens it)
            bool done = false;
            const long long t0 = clock64();
            while (!(done = tc::mbar_try_wait(mbar, phase)) && clock64() - t0 < g.wait_limit) {
            }
            phase ^= 1u;
            if (__syncthreads_or(!done)) {
                failed = true;
                if (t == 0) atomicExch(g.err, 1);
            }
            tc::fence_after_sync();
        }
        if (t == 0) g.sinfo[id] = info;
        if (!failed) {
            __syncthreads();   // the factorisation is done: its operand buffers are free
            TcRefineSmem& rf = *reinterpret_cast<TcRefineSmem*>(&sh.A[0][0][0]);
            if (info != 0) {   // singular in single precision (block-uniform)
                if (t == 0) {
                    g.iter[id] = -3;
                    g.fail_list[atomicAdd(g.fail_count, 1)] = id;
                }
            } else {
                if (w < (n >> 5)) tc_invert_block(sh.dblk[w], rf.inv[w][0], rf.inv[w][1], lane);
                __syncthreads();
                const int it = tc_refine_instance(g, id, t, lane, w, pos, trow, S, rf, keep);
                if (t == 0) {
                    g.iter[id] = it;
                    if (it < 0) g.fail_list[atomicAdd(g.fail_count, 1)] = id;
                }
            }
        }
        if (failed && t == 0) {
            // hand this instance and the rest of this block's share to the FP64 fallback
            for (int j = id; j < g.batch; j += gridDim.x) {
                g.iter[j] = -3;
                g.fail_list[atomicAdd(g.fail_count, 1)] = j;
            }
        }
        __syncthreads();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (w == 0) tc::tmem_dealloc(tbase, 512);
}

// The refinement's buffers overlay the L21 / U12 operand buffers (contiguous in TcLuSmem).
static_assert(offsetof(TcLuSmem, B) == sizeof(float) * 2 * 2 * 128 * 32, "operand buffers contiguous");
static_assert(sizeof(TcRefineSmem) <= offsetof(TcLuSmem, B) + sizeof(float) * 2 * kTcTrail * 32,
              "refinement buffers fit the operand buffers");

bool lu_tc_supported(int n) { return n >= 32 && n <= 256 && n % 32 == 0; }

size_t lu_tc_smem_bytes() { return sizeof(TcLuSmem) + 1024; }
// Two blocks of this kernel must never share an SM: each allocates all 512 TMEM columns.
static_assert(2 * (sizeof(TcLuSmem) + 1024) > 228 * 1024, "one tensor-core LU block per SM");

// Test hook state: > 0 replaces the completion-wait bound and suppresses the MMAs.
static std::atomic<long long> g_test_wait_limit{0};

magma_int_t lu_tc_launch(const TcLuArgs& in, cudaStream_t s) {
    TcLuArgs args = in;
    const long long hook = g_test_wait_limit.load(std::memory_order_relaxed);
    args.wait_limit = hook > 0 ? hook : (1ll << 33);
    args.issue_mma = hook > 0 ? 0 : 1;
    const int smem = (int)lu_tc_smem_bytes();
    ensure_dynamic_smem((const void*)lu_tf32x3_kernel, smem);
    const int grid = std::max(1, std::min(args.batch, device_sm_count()));
    lu_tf32x3_kernel<<<grid, kTcNT, smem, s>>>(args);
    return launch_status();
}

}  // namespace mb200

extern "C" void magma_b200_debug_tc_wait_limit(long long cycles) {
    mb200::g_test_wait_limit.store(cycles > 0 ? cycles : 0, std::memory_order_relaxed);
}
