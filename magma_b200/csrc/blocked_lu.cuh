// blocked_lu.cuh -- blocked right-looking LU (getrf) and blocked triangular
// solves (getrs) for one matrix per thread block, m <= NT rows.
//
// Replaces the reference's recursive-panel driver for these sizes
// (src/zgetrf_batched.cpp:222-351, src/zgetrf_panel_batched.cpp:128-243:
// ~90 launches per call, a cuBLAS stream loop for the trailing gemm) with one
// launch in which each thread block factors one matrix:
//
//   for each panel of NB columns (k0 = 0, NB, ...):
//     1. thread t loads row t of the panel into registers and the panel is
//        factored with the register steps of small_lu.cuh (pivot search over
//        the live rows, implicit row positions, rank-1 updates);
//     2. the panel is stored at the rows' new positions; rows displaced by
//        the panel's interchanges also move their columns left of the panel
//        (LAPACK applies DLASWP to A(:,1:k0));
//     3. for the trailing columns, in chunks of CW: the NB pivot rows are
//        gathered into shared memory and solved with L11 (U12 = L11^-1 A12,
//        one thread per column, in registers), then every other live row applies
//        A22 -= L21 U12 from its registers while moving to its new position,
//        and the U12 rows are stored.
//   After each panel the matrix is again in LAPACK's row order, so the next
//   panel starts with thread t = position t.
//
// Every element receives its updates as single fma's in increasing step
// order, exactly like the unblocked dgetf2 (DGER per step), so factors,
// pivots and info are bit-identical to the oracle restatement at every size.
#pragma once

#include "small_lu.cuh"

namespace mb200 {

template <typename T, int NB, int NT, int CW>
struct BlockedLuShared {
    SmallLuShared<T, NB, NT / 32> lu;
    T   L11[NB][NB + 1];
    T   U[NB][CW];
    int src[NB];
};

// U12 = L11^-1 A12 for column c of the staged pivot rows (sh.U[0..NB-1][c]),
// in groups of H rows held in registers: a group first takes the updates of
// the finished rows above it (read back from shared memory), then is solved
// in registers. Every entry receives fma(L11(r, rr), -U(rr, c), x) for rr
// ascending -- the unblocked order. Rows past the panel's last step hold
// unused values and are never stored.
template <typename T, int NB, int NT, int CW>
__device__ __forceinline__ void blocked_trsm_column(BlockedLuShared<T, NB, NT, CW>& sh, int c) {
    constexpr int H = 8;
    static_assert(NB % H == 0, "panel width must be a multiple of the TRSM group");
#pragma unroll 1
    for (int q0 = 0; q0 < NB; q0 += H) {
        T x[H];
#pragma unroll
        for (int r = 0; r < H; ++r) x[r] = sh.U[q0 + r][c];
#pragma unroll 2
        for (int rr = 0; rr < q0; ++rr) {
            const T u = sh.U[rr][c];
#pragma unroll
            for (int r = 0; r < H; ++r) x[r] = fma_rn(sh.L11[q0 + r][rr], -u, x[r]);
        }
        static_for<0, H>([&](auto rrc) {
            constexpr int rr = decltype(rrc)::value;
#pragma unroll
            for (int r = rr + 1; r < H; ++r) x[r] = fma_rn(sh.L11[q0 + r][q0 + rr], -x[rr], x[r]);
        });
#pragma unroll
        for (int r = 0; r < H; ++r) sh.U[q0 + r][c] = x[r];
    }
}

template <typename T, int NB, int NT, int CW, int CB>
__device__ void blocked_getrf(T* __restrict__ A, int m, int n, int lda, int* __restrict__ ipiv, int& info,
                              BlockedLuShared<T, NB, NT, CW>& sh) {
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x;
    const int kmax = min(m, n);
    info = 0;
    for (int k0 = 0; k0 < kmax; k0 += NB) {
        const int nbp = min(NB, kmax - k0);          // panel steps
        const int live = (tid >= k0 && tid < m);
        // ---- 1. panel factorisation in registers ----
        T a[NB];
#pragma unroll
        for (int c = 0; c < NB; ++c) a[c] = (live && c < nbp) ? A[tid + (size_t)(k0 + c) * lda] : T(0);
        int pos = (tid < m) ? tid : INT_MAX / 2;
        int my_ipiv = 0;
        lu_panel_steps<T, NB, NW>(a, m, nbp, nbp, k0, tid, pos, my_ipiv, info, sh.lu, ipiv == nullptr);
        if (ipiv && tid >= k0 && tid < k0 + nbp) ipiv[tid] = my_ipiv;
        const bool pivot_row = live && pos < k0 + nbp;
        const bool displaced = live && pos != tid;
        // ---- 2. store the panel at the new positions; L11 and pivot sources to smem ----
        if (live) {
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if (c < nbp) A[pos + (size_t)(k0 + c) * lda] = a[c];
        }
        if (pivot_row) {
#pragma unroll
            for (int c = 0; c < NB; ++c) sh.L11[pos - k0][c] = a[c];
            sh.src[pos - k0] = tid;
        }
        // Interchanges applied to the columns left of the panel. Only displaced
        // rows move: pivot rows (slot pos-k0) and the rows they pushed out of
        // positions k0..k0+nbp-1 (slot nbp + tid-k0); they are staged through
        // the (idle) U buffer, viewed as 2*NB slots of CW/2 columns.
        {
            constexpr int LW = CW / 2;
            T* stage = &sh.U[0][0];
            const int slot = pivot_row ? (pos - k0) : (nbp + tid - k0);
            for (int j0 = 0; j0 < k0; j0 += LW) {
                const int w = min(LW, k0 - j0);
                __syncthreads();
                if (displaced)
                    for (int c = 0; c < w; ++c) stage[slot * LW + c] = A[tid + (size_t)(j0 + c) * lda];
                __syncthreads();
                if (displaced)
                    for (int c = 0; c < w; ++c) A[pos + (size_t)(j0 + c) * lda] = stage[slot * LW + c];
            }
        }
        // ---- 3. trailing columns ----
        // A non-pivot row's own trailing entries are written only by itself, so the
        // next CB of them are loaded one group ahead (across the barriers) to hide
        // the load latency behind the current group's arithmetic.
        const bool upd = live && !pivot_row;
        T nxt[CB];
        auto prefetch = [&](int j) {
#pragma unroll
            for (int c = 0; c < CB; ++c) nxt[c] = (upd && j + c < n) ? A[tid + (size_t)(j + c) * lda] : T(0);
        };
        prefetch(k0 + nbp);
        for (int j0 = k0 + nbp; j0 < n; j0 += CW) {
            const int cw = min(CW, n - j0);
            __syncthreads();   // sU / L11 / src ready; previous chunk's readers done
            for (int idx = tid; idx < nbp * cw; idx += NT) {
                const int r = idx % nbp, c = idx / nbp;
                sh.U[r][c] = A[sh.src[r] + (size_t)(j0 + c) * lda];
            }
            __syncthreads();
            // U12 = L11^-1 A12, one thread per column, in two halves of H rows held in
            // registers; each entry gets its fma's in ascending step order.
            for (int c = tid; c < cw; c += NT) blocked_trsm_column<T, NB, NT, CW>(sh, c);
            __syncthreads();
            // A22 -= L21 U12 for the non-pivot live rows, stored at their new positions.
            // A row only ever overwrites the old row of a pivot (already gathered above),
            // so no barrier is needed between these loads and stores.
            if (upd) {
                for (int c0 = 0; c0 < cw; c0 += CB) {
                    T acc[CB];
#pragma unroll
                    for (int c = 0; c < CB; ++c) acc[c] = nxt[c];
                    prefetch(j0 + c0 + CB);
                    static_for<0, NB>([&](auto rc) {
                        constexpr int r = decltype(rc)::value;
                        if (r < nbp) {
                            const T l = a[r];
#pragma unroll
                            for (int c = 0; c < CB; ++c) acc[c] = fma_rn(l, -sh.U[r][c0 + c], acc[c]);
                        }
                    });
#pragma unroll
                    for (int c = 0; c < CB; ++c)
                        if (c0 + c < cw) A[pos + (size_t)(j0 + c0 + c) * lda] = acc[c];
                }
            }
            __syncthreads();   // every displaced row has read its old row before U12 lands there
            for (int idx = tid; idx < nbp * cw; idx += NT) {
                const int r = idx % nbp, c = idx / nbp;
                A[k0 + r + (size_t)(j0 + c) * lda] = sh.U[r][c];
            }
        }
        __syncthreads();   // panel k0 complete before the next panel reads rows
    }
}

}  // namespace mb200
