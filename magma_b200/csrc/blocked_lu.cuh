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
//        A22 -= L21 U12 while moving to its new position -- in FP64 on the tensor
//        cores (mma.sync m8n8k4 .f64: each warp's 32 rows as four 8-row groups,
//        8-column tiles, the multipliers as A fragments read back from the stored
//        panel), in FP32 from registers -- and the U12 rows are stored.
//   After each panel the matrix is again in LAPACK's row order, so the next
//   panel starts with thread t = position t.
//
// Every element receives its updates as single fma's in increasing step
// order, exactly like the unblocked dgetf2 (DGER per step), so factors,
// pivots and info are bit-identical to the oracle restatement at every size.
// This holds on the tensor cores too: an m8n8k4 FP64 MMA gives each element the
// four products as a chain of fma's in ascending k, each rounded (measured on
// B200 against the fma chain: 1.28 M of 1.28 M elements equal), and the k-steps
// are issued in ascending order.
#pragma once

#include "small_lu.cuh"
#include <type_traits>

namespace mb200 {

template <typename T, int NB, int NT, int CW, bool DMMA = false>
struct BlockedLuShared {
    SmallLuShared<T, NB, NT / 32> lu;
    T   L11[NB][NB + 1];
    // pivot rows' trailing columns, then U12; rows padded to CW + 1 so that a warp
    // reading one column across 32 rows (gather, U12 store) hits every bank pair twice
    T   U[NB][CW + 1];
    int src[NB];
    // DMMA update: the panel's multipliers as tensor-core A fragments,
    // [warp][row group][k-step][lane] (each lane reads its own 8 bytes)
    T   af[DMMA ? NT / 32 : 1][4][DMMA ? NB / 4 : 1][32];
};

// U12 = L11^-1 A12 for column c of the staged pivot rows (sh.U[0..NB-1][c]),
// in groups of H rows held in registers: a group first takes the updates of
// the finished rows above it (read back from shared memory), then is solved
// in registers. Every entry receives fma(L11(r, rr), -U(rr, c), x) for rr
// ascending -- the unblocked order. Rows past the panel's last step hold
// unused values and are never stored.
template <typename T, int NB, int NT, int CW, bool DMMA>
__device__ __forceinline__ void blocked_trsm_column(BlockedLuShared<T, NB, NT, CW, DMMA>& sh, int c) {
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

// One FP64 tensor-core step D = A B + D on an 8x8 tile (A 8x4 row-major, B 4x8
// column-major; lane l holds A(l/4, l%4), B(l%4, l/4), D(l/4, 2(l%4) .. +1)). Each
// element of D receives fma(a(i,0), b(0,j), d) then k = 1, 2, 3 in ascending order,
// rounded after every step -- the same operations as four single fma's in k order,
// which keeps the blocked update bit-identical to the unblocked elimination.
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// A22 -= L21 U12 for the warp's 32 rows and the chunk's cw columns on the FP64
// tensor cores. The A fragment of row group g (rows 8g..8g+7 of the warp) and k-step
// s (panel columns 4s..4s+3) is the row's multiplier, read from the panel stored at
// the row's new position rpos[g]; 0 for rows that take no update and for columns
// past the panel's steps. Row 8g + l/4 of the warp
// reads its C entries at its current position and writes them to rpos[g] (rupd[g]
// false: not read, not written). B = -U12 from shared memory, 0 past the chunk. The
// C entries of the next 8-column tile are loaded while the current tile computes.
template <int NB, int NT, int CW>
__device__ __forceinline__ void blocked_update_dmma(double* A, int lda, int k0, int j0, int cw, int nbp,
                                                    const int (&rpos)[4], const bool (&rupd)[4],
                                                    const double (&U)[NB][CW + 1], const double (&af)[4][NB / 4][32],
                                                    int tid) {
    constexpr int KS = NB / 4;
    const int lane = tid & 31;
    const int row0 = (tid & ~31) + (lane >> 2);   // warp's first row + this lane's row in a group
    const int q = lane & 3;
    const int ks = (nbp + 3) / 4;                         // k-steps with a panel column
    bool gact[4];                                         // groups with a row to update
#pragma unroll
    for (int g = 0; g < 4; ++g) gact[g] = __any_sync(kFullMask, rupd[g]);
    if (!(gact[0] || gact[1] || gact[2] || gact[3])) return;   // every row of the warp is done
    double cn[4][2];
    auto load_c = [&](int jt) {
        const int c0 = jt + 2 * q;
        const double* src0 = A + (size_t)(j0 + c0) * lda;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const int r = row0 + 8 * g;                   // the row's position before this panel
            cn[g][0] = (c0 < cw && rupd[g]) ? src0[r] : 0.0;
            cn[g][1] = (c0 + 1 < cw && rupd[g]) ? src0[r + lda] : 0.0;
        }
    };
    load_c(0);
#pragma unroll 1
    for (int jt = 0; jt < cw; jt += 8) {
        double cc[4][2];
#pragma unroll
        for (int g = 0; g < 4; ++g) { cc[g][0] = cn[g][0]; cc[g][1] = cn[g][1]; }
        if (jt + 8 < cw) load_c(jt + 8);
        double b[KS];
        const int cb = jt + (lane >> 2);                  // B column of this lane
#pragma unroll
        for (int s = 0; s < KS; ++s) b[s] = (cb < cw && 4 * s + q < nbp) ? -U[4 * s + q][cb] : 0.0;
#pragma unroll
        for (int s = 0; s < KS; ++s) {
            if (s < ks) {
#pragma unroll
                for (int g = 0; g < 4; ++g)
                    if (gact[g]) dmma_884(cc[g][0], cc[g][1], af[g][s][lane], b[s]);
            }
        }
        const int c0 = jt + 2 * q;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            if (rupd[g]) {
                double* dst = A + (size_t)(j0 + c0) * lda + rpos[g];
                if (c0 < cw) dst[0] = cc[g][0];
                if (c0 + 1 < cw) dst[lda] = cc[g][1];
            }
        }
    }
}

template <typename T, int NB, int NT, int CW, int CB, bool DMMA, typename Team = BlockTeam>
__device__ void blocked_getrf(T* __restrict__ A, int m, int n, int lda, int* __restrict__ ipiv, int& info,
                              BlockedLuShared<T, NB, NT, CW, DMMA>& sh, const Team& team = Team{}) {
    constexpr int NW = NT / 32;
    const int tid = team.tid();
    auto sync = [&] { team.sync(); };
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
        lu_panel_steps<T, NB, NW>(a, m, nbp, nbp, k0, tid, pos, my_ipiv, info, sh.lu, ipiv == nullptr, sync);
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
                team.sync();
                if (displaced)
                    for (int c = 0; c < w; ++c) stage[slot * LW + c] = A[tid + (size_t)(j0 + c) * lda];
                team.sync();
                if (displaced)
                    for (int c = 0; c < w; ++c) A[pos + (size_t)(j0 + c) * lda] = stage[slot * LW + c];
            }
        }
        // ---- 3. trailing columns ----
        // A non-pivot row's own trailing entries are written only by itself, so the
        // next CB of them are loaded one group ahead (across the barriers) to hide
        // the load latency behind the current group's arithmetic.
        const bool upd = live && !pivot_row;
        constexpr bool kDmma = DMMA && std::is_same<T, double>::value;
        // FP64: the update runs on the tensor cores; the A fragments (the rows'
        // multipliers) of the warp's four row groups go to shared memory once per
        // panel, gathered by shuffles.
        int rpos[4];
        bool rupd[4];
        if constexpr (kDmma) {
            const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                const int srcl = 8 * g + (lane >> 2);
                rpos[g] = __shfl_sync(kFullMask, pos, srcl);
                rupd[g] = __shfl_sync(kFullMask, (int)upd, srcl) != 0;
#pragma unroll
                for (int s = 0; s < NB / 4; ++s) {
                    double v = 0.0;
#pragma unroll
                    for (int qq = 0; qq < 4; ++qq) {
                        const double x = __shfl_sync(kFullMask, (double)a[4 * s + qq], srcl);
                        if ((lane & 3) == qq) v = x;
                    }
                    sh.af[warp][g][s][lane] = (rupd[g] && 4 * s + (lane & 3) < nbp) ? v : 0.0;
                }
            }
        }
        T nxt[CB];
        auto prefetch = [&](int j) {
            if constexpr (kDmma) return;
#pragma unroll
            for (int c = 0; c < CB; ++c) nxt[c] = (upd && j + c < n) ? A[tid + (size_t)(j + c) * lda] : T(0);
        };
        prefetch(k0 + nbp);
        for (int j0 = k0 + nbp; j0 < n; j0 += CW) {
            const int cw = min(CW, n - j0);
            team.sync();   // sU / L11 / src ready; previous chunk's readers done
            for (int idx = tid; idx < nbp * cw; idx += NT) {
                const int r = idx % nbp, c = idx / nbp;
                sh.U[r][c] = A[sh.src[r] + (size_t)(j0 + c) * lda];
            }
            team.sync();
            // U12 = L11^-1 A12, one thread per column, in two halves of H rows held in
            // registers; each entry gets its fma's in ascending step order.
            for (int c = tid; c < cw; c += NT) blocked_trsm_column<T, NB, NT, CW, DMMA>(sh, c);
            team.sync();
            // A22 -= L21 U12 for the non-pivot live rows, stored at their new positions.
            // A row only ever overwrites the old row of a pivot (already gathered above),
            // so no barrier is needed between these loads and stores.
            if constexpr (kDmma) {
                blocked_update_dmma<NB, NT, CW>(reinterpret_cast<double*>(A), lda, k0, j0, cw, nbp, rpos, rupd,
                                                reinterpret_cast<const double(&)[NB][CW + 1]>(sh.U),
                                                reinterpret_cast<const double(&)[4][NB / 4][32]>(sh.af[tid >> 5]), tid);
            } else if (upd) {
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
            team.sync();   // every displaced row has read its old row before U12 lands there
            for (int idx = tid; idx < nbp * cw; idx += NT) {
                const int r = idx % nbp, c = idx / nbp;
                A[k0 + r + (size_t)(j0 + c) * lda] = sh.U[r][c];
            }
        }
        team.sync();   // panel k0 complete before the next panel reads rows
    }
}

}  // namespace mb200
