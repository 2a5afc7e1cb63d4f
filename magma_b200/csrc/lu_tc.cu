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
    float L11[32][33];
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
__device__ __forceinline__ void tc_trsm_column(TcLuSmem& sh, int c) {
#pragma unroll 1
    for (int q0 = 0; q0 < 32; q0 += 8) {
        float x[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) x[r] = sh.Ug[q0 + r][c];
        for (int rr = 0; rr < q0; ++rr) {
            const float u = sh.Ug[rr][c];
#pragma unroll
            for (int r = 0; r < 8; ++r) x[r] = fmaf(sh.L11[q0 + r][rr], -u, x[r]);
        }
        static_for<0, 8>([&](auto rc) {
            constexpr int rr = decltype(rc)::value;
#pragma unroll
            for (int r = rr + 1; r < 8; ++r) x[r] = fmaf(sh.L11[q0 + r][q0 + rr], -x[rr], x[r]);
        });
#pragma unroll
        for (int r = 0; r < 8; ++r) sh.Ug[q0 + r][c] = x[r];
    }
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
    for (int id = blockIdx.x; id < g.batch && !failed; id += gridDim.x) {
        const double* A = g.dA[id];
        float* S = g.SA + (size_t)id * n * n;
        // ---- 1. FP64 row -> FP32 TMEM, row sums, overflow ----
        double rs = 0.0;
        bool ovf = false;
        for (int c0 = 0; c0 < n; c0 += 32) {
            float v[32];
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const double a = (t < n) ? A[t + (size_t)(c0 + c) * g.lda] : 0.0;
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
            // the next instance's FP64 columns into L2 while this one finishes (thread t:
            // column t), so its conversion reads from L2 instead of HBM
            if (k0 == (n >= 64 ? n - 64 : 0) && id + (int)gridDim.x < g.batch && t < n)
                prefetch_l2(g.dA[id + gridDim.x] + (size_t)t * g.lda, unsigned(n) * 8u);
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
                for (int c = 0; c < 32; ++c) sh.L11[pos - k0][c] = a[c];
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
            if (piv) {
#pragma unroll
                for (int c = 0; c < 32; ++c) S[pos + (size_t)(k0 + c) * n] = a[c];
            }
            tc::wait_st();
            __syncthreads();
            if (ncols <= 0) break;
            for (int c = t; c < ncols; c += kTcNT) tc_trsm_column(sh, c);
            __syncthreads();
            // U12 rows to the output, and the split B operand
            for (int idx = t; idx < 32 * ncols; idx += kTcNT) {
                const int r = idx & 31, c = idx >> 5;
                S[(k0 + r) + (size_t)(k0 + 32 + c) * n] = sh.Ug[r][c];
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
        if (!failed) {
            // every row's L entries left of the panel that chose it, at its final position
            const int myk = (t < n) ? (pos & ~31) : 0;
            const int wk = (int)__reduce_max_sync(kFullMask, (unsigned)myk);
            for (int c0 = 0; c0 < wk; c0 += 32) {
                float v[32];
                tc::tmem_ld32(trow + c0, v);
                tc::wait_ld();
                if (c0 < myk) {
#pragma unroll
                    for (int c = 0; c < 32; ++c) S[pos + (size_t)(c0 + c) * n] = v[c];
                }
            }
        }
        if (t == 0) g.sinfo[id] = info;
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
