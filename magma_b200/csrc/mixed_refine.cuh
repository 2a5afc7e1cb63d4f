// mixed_refine.cuh -- the refinement stage of the batched mixed-precision solve:
// one thread block per instance, thread t = row t, up to NT rows.
//
// Each refinement pass solves L U c = P r in single precision and updates the
// FP64 solution and residual. The single-precision solve only has to be
// accurate to working precision (its result is a correction), so it uses the
// explicit inverses of the 32x32 diagonal blocks of L and U, as the reference's
// batched trsm does (trtri of the diagonal blocks + gemm, src/zgetrs_batched.cpp
// :178-266): the inverses are formed once per instance (one warp per block, one
// lane per column), and a block step of the solve is then a product with the
// inverse by the warp that owns the block plus an update of the other rows --
// one barrier per 32-row block instead of 32 dependent steps.
#pragma once

#include "small_lu.cuh"
#include <cfloat>

namespace mb200 {

template <int NT, int R>
struct RefineSmem {
    static constexpr int NBLK = NT / 32;
    float  inv[NBLK][2][32][33];   // [block][0: L^-1 (unit lower), 1: U^-1][row][col]
    float  sx[2][32][R];           // solved values of the current block (double-buffered)
    float  sb[NBLK][32][R];        // per-warp staging of a block's right-hand sides
    float  xch[NT][R];             // row permutation exchange
    double xs[NT][R];              // FP64 solution, shared for the residual
    double red[2][NBLK][R];
    int    ipiv[NT];
};

// Inverse of the diagonal block J of the factors in SA (n x n, column-major),
// computed by one warp: lane j forms column j of L_JJ^-1 and of U_JJ^-1.
// Rows/columns past n are treated as the identity.
template <int NT, int R>
__device__ __forceinline__ void invert_diag_block(const float* __restrict__ SA, int n, int J, int lane,
                                                  RefineSmem<NT, R>& sh) {
    const int j0 = J * 32;
    float (&T)[32][33] = sh.inv[J][1];   // staging: the raw diagonal block, then U^-1
#pragma unroll 4
    for (int k = 0; k < 32; ++k)
        T[lane][k] = (j0 + lane < n && j0 + k < n) ? SA[j0 + lane + (size_t)(j0 + k) * n]
                                                   : (lane == k ? 1.0f : 0.0f);
    __syncwarp();
    float x[32];
    // L^-1, column `lane`: forward substitution on e_lane (unit diagonal)
    static_for<0, 32>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        float s = (i == lane) ? 1.0f : 0.0f;
#pragma unroll
        for (int k = 0; k < i; ++k) s = fmaf(-T[i][k], x[k], s);
        x[i] = (i < lane) ? 0.0f : s;
    });
#pragma unroll
    for (int i = 0; i < 32; ++i) sh.inv[J][0][i][lane] = x[i];
    // U^-1, column `lane`: backward substitution on e_lane
    static_for<0, 32>([&](auto ic) {
        constexpr int i = 31 - decltype(ic)::value;
        float s = (i == lane) ? 1.0f : 0.0f;
#pragma unroll
        for (int k = i + 1; k < 32; ++k) s = fmaf(-T[i][k], x[k], s);
        x[i] = (i > lane) ? 0.0f : s / T[i][i];
    });
    __syncwarp();   // every lane has read the raw block before it is overwritten
#pragma unroll
    for (int i = 0; i < 32; ++i) T[i][lane] = x[i];
    __syncwarp();
}

// Solves L U c = b in single precision for the R right-hand sides in f (thread t
// holds row t of P*b; on return row t of c). Warp J owns the rows of block J.
template <int NT, int R>
__device__ __forceinline__ void refine_solve(const float* __restrict__ SA, int n, float (&f)[R],
                                             RefineSmem<NT, R>& sh) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int nblk = (n + 31) / 32;
    // L2 prefetch of the panel a later block step reads: columns of block J2, the rows
    // below the block (forward sweep) or above it (backward sweep); lane k takes column k.
    auto prefetch_panel = [&](int J2, bool below) {
        const int col = J2 * 32 + lane;
        const int r0 = below ? (J2 + 1) * 32 : 0, r1 = below ? n : J2 * 32;
        if (col < n && r1 > r0) prefetch_l2(SA + (size_t)col * n + r0, (unsigned)(r1 - r0) * 4u);
    };
    // block step of the warp that owns block J: f_J <- inv * f_J, published in sx[buf]
    auto diag_step = [&](int J, int which, int buf) {
#pragma unroll
        for (int r = 0; r < R; ++r) sh.sb[w][lane][r] = f[r];
        __syncwarp();
        float x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = 0.0f;
#pragma unroll 8
        for (int k = 0; k < 32; ++k) {
            const float l = sh.inv[J][which][lane][k];
#pragma unroll
            for (int r = 0; r < R; ++r) x[r] = fmaf(l, sh.sb[w][k][r], x[r]);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            f[r] = x[r];
            sh.sx[buf][lane][r] = x[r];
        }
    };
    // forward: unit lower L, blocks ascending; rows below the block apply its update
    for (int J = 0; J < nblk; ++J) {
        const int j0 = J * 32, buf = J & 1;
        if (w == (J == 0 ? 1 : 0)) {   // a warp that is idle in this step prefetches the next one's panel
            if (J + 1 < nblk) prefetch_panel(J + 1, true);
            else prefetch_panel(J, false);
        }
        float lv[32];
        const bool below = (w > J && t < n);
        if (below) {
#pragma unroll
            for (int k = 0; k < 32; ++k) lv[k] = (j0 + k < n) ? SA[t + (size_t)(j0 + k) * n] : 0.0f;
        }
        if (w == J) diag_step(J, 0, buf);
        __syncthreads();
        if (below) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
#pragma unroll
                for (int r = 0; r < R; ++r) f[r] = fmaf(-lv[k], sh.sx[buf][k][r], f[r]);
            }
        }
    }
    // backward: U, blocks descending; rows above the block apply its update
    for (int J = nblk - 1; J >= 0; --J) {
        const int j0 = J * 32, buf = (2 * nblk - 1 - J) & 1;
        if (J > 0 && w == (J == nblk - 1 ? 0 : nblk - 1)) prefetch_panel(J - 1, false);
        float uv[32];
        const bool above = (w < J);
        if (above) {
#pragma unroll
            for (int k = 0; k < 32; ++k) uv[k] = (j0 + k < n) ? SA[t + (size_t)(j0 + k) * n] : 0.0f;
        }
        if (w == J) diag_step(J, 1, buf);
        __syncthreads();
        if (above) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
#pragma unroll
                for (int r = 0; r < R; ++r) f[r] = fmaf(-uv[k], sh.sx[buf][k][r], f[r]);
            }
        }
    }
}

// Block-wide maxima of v and w per right-hand side (every thread gets them).
template <int NT, int R>
__device__ __forceinline__ void refine_max2(double (&v)[R], double (&w)[R], RefineSmem<NT, R>& sh) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        for (int off = 16; off > 0; off >>= 1) {
            v[r] = fmax(v[r], __shfl_xor_sync(kFullMask, v[r], off));
            w[r] = fmax(w[r], __shfl_xor_sync(kFullMask, w[r], off));
        }
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            sh.red[0][threadIdx.x >> 5][r] = v[r];
            sh.red[1][threadIdx.x >> 5][r] = w[r];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        v[r] = 0.0;
        w[r] = 0.0;
        for (int k = 0; k < NT / 32; ++k) {
            v[r] = fmax(v[r], sh.red[0][k][r]);
            w[r] = fmax(w[r], sh.red[1][k][r]);
        }
    }
}

}  // namespace mb200
