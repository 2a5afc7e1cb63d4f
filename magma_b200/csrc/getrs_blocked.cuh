// getrs_blocked.cuh -- blocked triangular solves with the LU factors of one
// matrix per thread block (n <= NT), R right-hand sides at a time.
//
// Replaces the reference's getrs for these sizes (src/zgetrs_batched.cpp:87-273:
// dlaswp_rowserial, then trsv for one RHS or trtri-of-diagonal-blocks + gemm
// for several) by one launch. Thread t owns row t of the right-hand sides. The
// rows are swept in 32-row blocks: the warp that owns a block solves its
// diagonal block with warp-level barriers, then every thread below (or above)
// applies the block's contribution reading L (or U) once, coalesced by column.
// Each entry receives its updates as single fma's in the order of reference
// BLAS dtrsm (k ascending for L, descending for U), so NoTrans solutions are
// bit-identical to the oracle; the transposed L solve uses descending order.
#pragma once

#include "small_lu.cuh"

namespace mb200 {

template <typename T, int NT, int R>
struct BlockedRsShared {
    T   x[NT][R];       // permutation exchange
    T   sb[32][R];      // solved values of the current 32-row block
    T   D[32][33];      // the current 32x32 diagonal block
    int ipiv[NT];
};

// idx = where original row t of B sits after DLASWP (forward or inverse order).
__device__ __forceinline__ int laswp_target(const int* s_ipiv, int n, int t, bool inverse) {
    int idx = t;
    if (!inverse) {
        for (int k = 0; k < n; ++k) {
            const int p = s_ipiv[k] - 1;
            idx = (idx == k) ? p : (idx == p) ? k : idx;
        }
    } else {
        for (int k = n - 1; k >= 0; --k) {
            const int p = s_ipiv[k] - 1;
            idx = (idx == k) ? p : (idx == p) ? k : idx;
        }
    }
    return idx;
}

template <typename T, int NT, int R, typename Team>
__device__ __forceinline__ void permute_rows(T (&b)[R], int n, int t, int idx, BlockedRsShared<T, NT, R>& sh,
                                             const Team& team) {
    team.sync();
    if (t < n) {
#pragma unroll
        for (int r = 0; r < R; ++r) sh.x[idx][r] = b[r];
    }
    team.sync();
    if (t < n) {
#pragma unroll
        for (int r = 0; r < R; ++r) b[r] = sh.x[t][r];
    }
}


// Warp `J` stages the diagonal block A[j0:j1, j0:j1] into shared memory. The loads go
// out unconditionally (clamped inside the block), 8 at a time, so they overlap.
template <typename T, int NT, int R>
__device__ __forceinline__ void stage_diag(const T* __restrict__ A, int lda, int j0, int j1, int t,
                                           BlockedRsShared<T, NT, R>& sh) {
    const int lane = t & 31, cnt = j1 - j0;
    const int li = j0 + min(lane, cnt - 1);
#pragma unroll
    for (int c0 = 0; c0 < 32; c0 += 8) {
        T v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = A[li + (size_t)(j0 + min(c0 + c, cnt - 1)) * lda];
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c0 + c < cnt && lane < cnt) sh.D[lane][c0 + c] = v[c];
    }
    __syncwarp();
}

// op(A) X = B for one matrix; A holds the getrf factors, B is overwritten.
template <typename T, int NT, int R, typename Team = BlockTeam>
__device__ void blocked_getrs(bool trans, const T* __restrict__ A, int n, int lda, const int* __restrict__ ipiv,
                              T* __restrict__ B, int nrhs, int ldb, BlockedRsShared<T, NT, R>& sh,
                              const Team& team = Team{}) {
    const int t = team.tid();
    for (int k = t; k < n; k += NT) sh.ipiv[k] = ipiv ? ipiv[k] : k + 1;   // no pivots: identity
    team.sync();
    const int fwd_idx = (t < n) ? laswp_target(sh.ipiv, n, t, false) : t;
    const int inv_idx = (t < n) ? laswp_target(sh.ipiv, n, t, true) : t;
    const int nblk = (n + 31) / 32;
    for (int c0 = 0; c0 < nrhs; c0 += R) {
        T b[R];
#pragma unroll
        for (int r = 0; r < R; ++r) b[r] = (t < n && c0 + r < nrhs) ? B[t + (size_t)(c0 + r) * ldb] : T(0);
        if (!trans) {
            permute_rows<T, NT, R>(b, n, t, fwd_idx, sh, team);
            // ---- L (unit lower), blocks ascending ----
            for (int J = 0; J < nblk; ++J) {
                const int j0 = J * 32, j1 = min(n, j0 + 32);
                team.sync();
                if ((t >> 5) == J) {   // the warp that owns rows j0..j1-1 solves the diagonal block
                    stage_diag<T, NT, R>(A, lda, j0, j1, t, sh);
                    const int lane = t & 31, cnt = j1 - j0;
                    static_for<0, 32>([&](auto kc) {   // steps unrolled: no loop overhead on the chain
                        constexpr int k = decltype(kc)::value;
                        if (k >= cnt) return;
                        if (lane == k) {
#pragma unroll
                            for (int r = 0; r < R; ++r) sh.sb[k][r] = b[r];
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
                if (t >= j1 && t < n) {
#pragma unroll
                    for (int kk = 0; kk < 32; ++kk) {
                        if (j0 + kk < j1) {
                            const T l = A[t + (size_t)(j0 + kk) * lda];
#pragma unroll
                            for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.sb[kk][r], l, b[r]);
                        }
                    }
                }
            }
            // ---- U (non-unit upper), blocks descending ----
            for (int J = nblk - 1; J >= 0; --J) {
                const int j0 = J * 32, j1 = min(n, j0 + 32);
                team.sync();
                if ((t >> 5) == J) {
                    stage_diag<T, NT, R>(A, lda, j0, j1, t, sh);
                    const int lane = t & 31, cnt = j1 - j0;
                    static_for<0, 32>([&](auto kc) {
                        constexpr int k = 31 - decltype(kc)::value;
                        if (k >= cnt) return;
                        if (lane == k) {
                            const T d = sh.D[k][k];
#pragma unroll
                            for (int r = 0; r < R; ++r) {
                                b[r] = b[r] / d;
                                sh.sb[k][r] = b[r];
                            }
                        }
                        __syncwarp();
                        if (lane < k) {
                            const T u = sh.D[lane][k];
#pragma unroll
                            for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.sb[k][r], u, b[r]);
                        }
                    });
                }
                team.sync();
                if (t < j0) {
#pragma unroll
                    for (int kk = 31; kk >= 0; --kk) {
                        if (j0 + kk < j1) {
                            const T u = A[t + (size_t)(j0 + kk) * lda];
#pragma unroll
                            for (int r = 0; r < R; ++r) b[r] = fma_rn(-sh.sb[kk][r], u, b[r]);
                        }
                    }
                }
            }
        } else {
            // ---- U^T (non-unit lower), blocks ascending: y_k = b_k / U(k,k), b_i -= U(k,i) y_k ----
            for (int J = 0; J < nblk; ++J) {
                const int j0 = J * 32, j1 = min(n, j0 + 32);
                team.sync();
                if ((t >> 5) == J) {
                    stage_diag<T, NT, R>(A, lda, j0, j1, t, sh);
                    const int lane = t & 31, cnt = j1 - j0;
                    static_for<0, 32>([&](auto kc) {
                        constexpr int k = decltype(kc)::value;
                        if (k >= cnt) return;
                        if (lane == k) {
                            const T d = sh.D[k][k];
#pragma unroll
                            for (int r = 0; r < R; ++r) {
                                b[r] = b[r] / d;
                                sh.sb[k][r] = b[r];
                            }
                        }
                        __syncwarp();
                        if (lane > k && lane < cnt) {
                            const T u = sh.D[k][lane];
#pragma unroll
                            for (int r = 0; r < R; ++r) b[r] = fma_rn(-u, sh.sb[k][r], b[r]);
                        }
                    });
                }
                team.sync();
                if (t >= j1 && t < n) {
#pragma unroll
                    for (int kk = 0; kk < 32; ++kk) {
                        if (j0 + kk < j1) {
                            const T u = A[j0 + kk + (size_t)t * lda];
#pragma unroll
                            for (int r = 0; r < R; ++r) b[r] = fma_rn(-u, sh.sb[kk][r], b[r]);
                        }
                    }
                }
            }
            // ---- L^T (unit upper), blocks descending ----
            for (int J = nblk - 1; J >= 0; --J) {
                const int j0 = J * 32, j1 = min(n, j0 + 32);
                team.sync();
                if ((t >> 5) == J) {
                    stage_diag<T, NT, R>(A, lda, j0, j1, t, sh);
                    const int lane = t & 31, cnt = j1 - j0;
                    static_for<0, 32>([&](auto kc) {
                        constexpr int k = 31 - decltype(kc)::value;
                        if (k >= cnt) return;
                        if (lane == k) {
#pragma unroll
                            for (int r = 0; r < R; ++r) sh.sb[k][r] = b[r];
                        }
                        __syncwarp();
                        if (lane < k) {
                            const T l = sh.D[k][lane];
#pragma unroll
                            for (int r = 0; r < R; ++r) b[r] = fma_rn(-l, sh.sb[k][r], b[r]);
                        }
                    });
                }
                team.sync();
                if (t < j0) {
#pragma unroll
                    for (int kk = 31; kk >= 0; --kk) {
                        if (j0 + kk < j1) {
                            const T l = A[j0 + kk + (size_t)t * lda];
#pragma unroll
                            for (int r = 0; r < R; ++r) b[r] = fma_rn(-l, sh.sb[kk][r], b[r]);
                        }
                    }
                }
            }
            permute_rows<T, NT, R>(b, n, t, inv_idx, sh, team);
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
