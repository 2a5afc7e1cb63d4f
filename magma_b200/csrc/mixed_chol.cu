// mixed_chol.cu -- variable-size batched mixed-precision Cholesky solve
// (magma_dsposv_vbatched): FP32 potrf, FP64 iterative refinement, FP64 fallback.
//
// Per instance this follows magma_dsposv_gpu (src/zcposv_gpu.cpp:134-330) with
// uplo = Lower, the only form MAGMA's variable-size Cholesky supports:
//   Anrm = ||A||_inf of the symmetric matrix (zlanhe, :198), cte = Anrm*eps*sqrt(n)
//   SA = single(A) (zlat2c, :209); overflow -> iter = -2, fallback
//   SA = L L^T in single (cpotrf, :216); info > 0 -> iter = -3, fallback
//   X = SA^-1 B; R = B - A X (symmetric, double); refinement loop as dsgesv
//   (ITERMAX 30; no convergence -> iter = -31); fallback: dpotrf + dpotrs in FP64.
// As in magma_dsgesv_batched, refinement also stops (iter = -31) when the residual
// ratio fails to halve over two consecutive iterations.
//
// Batched form: the caller passes per-instance single-precision workspaces
// (dworks_array[i], at least n_i*(n_i + nrhs_i) floats, the reference's dworks
// size); the library's own workspace holds only per-instance scalars and the
// bucket lists. Instances are bucketed by n on the device; the conversion,
// refinement and fallback kernels walk the bucket lists, the FP32 and FP64
// factorisations reuse the Cholesky bucket kernels. No host synchronisation in
// the _max_nocheck form.
#include "internal.h"
#include "chol_launch.h"
#include "tuning.h"
#include "small_lu.cuh"
#include "vbatched.h"
#include <algorithm>
#include <cfloat>

namespace mb200 {

constexpr int kCholItermax = 30;

struct CholMixedWs {
    int* sinfo;      // FP32 potrf info
    double* anrm;    // ||A||_inf
    int* fkey;       // n_i for instances that need the FP64 fallback, else 0
    int* ldsa;       // leading dimension of SA_i (= n_i), batch + 1 entries
};

// ---- 1. SA = single(lower(A)), symmetric ||A||_inf, overflow check ----
// One block per instance; thread t = row t. Row sums of |A| use the stored lower
// triangle twice: row part sum_{j<=i} |a_ij| (thread per row, coalesced by column)
// plus column part sum_{k>i} |a_ki| (one warp per column).
template <int NT>
__global__ void __launch_bounds__(NT)
dlat2s_norm_vkernel(WorkList wl, const int* n_arr, double** dA_array, const int* ldda, float** dS_array,
                    CholMixedWs ws, int* iter_array) {
    __shared__ double colpart[NT];
    __shared__ double red[NT / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (int it = blockIdx.x; it < wl.size(); it += gridDim.x) {
        const int id = wl.at(it);
        const int n = n_arr[id], lda = ldda[id];
        const double* A = dA_array[id];
        float* SA = dS_array[id];
        bool overflow = false;
        double rowpart = 0.0;
        if (t < n) {
            for (int j = 0; j <= t; ++j) {
                const double a = A[t + (size_t)j * lda];
                rowpart += fabs(a);
                overflow |= !(fabs(a) <= (double)FLT_MAX);
                SA[t + (size_t)j * n] = (float)a;
            }
        }
        for (int c = w; c < n; c += NT / 32) {
            double s = 0.0;
            for (int k = c + 1 + lane; k < n; k += 32) s += fabs(A[k + (size_t)c * lda]);
            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(kFullMask, s, off);
            if (lane == 0) colpart[c] = s;
        }
        __syncthreads();
        double rs = (t < n) ? rowpart + colpart[t] : 0.0;
        for (int off = 16; off > 0; off >>= 1) rs = fmax(rs, __shfl_xor_sync(kFullMask, rs, off));
        if (lane == 0) red[w] = rs;
        const int ovf = __syncthreads_or(overflow);
        if (t == 0) {
            double m = 0.0;
            for (int k = 0; k < NT / 32; ++k) m = fmax(m, red[k]);
            ws.anrm[id] = m;
            ws.ldsa[id] = n;
            iter_array[id] = ovf ? -2 : 0;
            ws.fkey[id] = ovf ? n : 0;
        }
        __syncthreads();
    }
}

// ---- 2. refinement: one block per instance, thread t = row t, NT >= n ----
template <int NT, int R>
struct CholRefineSmem {
    static constexpr int NBLK = NT / 32;
    float  inv[NBLK][32][33];      // L_JJ^-1 of each 32x32 diagonal block
    float  sx[2][32][R];           // solved values of the current block (double-buffered)
    float  sb[NBLK][32][R];        // per-warp staging of a block's right-hand sides
    double xs[NT][R];              // FP64 solution, shared for the residual
    double red[2][NBLK][R];
};

// L_JJ^-1 (lower, non-unit) of diagonal block J of SA, by warp J: lane j forms column j.
template <int NT, int R>
__device__ __forceinline__ void chol_invert_diag_block(const float* __restrict__ SA, int n, int J, int lane,
                                                       CholRefineSmem<NT, R>& sh) {
    const int j0 = J * 32;
    float (&T)[32][33] = sh.inv[J];
#pragma unroll 4
    for (int k = 0; k < 32; ++k)
        T[lane][k] = (j0 + lane < n && j0 + k < n) ? (k <= lane ? SA[j0 + lane + (size_t)(j0 + k) * n] : 0.0f)
                                                   : (lane == k ? 1.0f : 0.0f);
    __syncwarp();
    float x[32];
    static_for<0, 32>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        float s = (i == lane) ? 1.0f : 0.0f;
#pragma unroll
        for (int k = 0; k < i; ++k) s = fmaf(-T[i][k], x[k], s);
        x[i] = (i < lane) ? 0.0f : s / T[i][i];
    });
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 32; ++i) T[i][lane] = x[i];
    __syncwarp();
}

// L L^T c = b in single precision for the R right-hand sides in f (thread t = row t).
template <int NT, int R>
__device__ __forceinline__ void chol_refine_solve(const float* __restrict__ SA, int n, float (&f)[R],
                                                  CholRefineSmem<NT, R>& sh) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int nblk = (n + 31) / 32;
    auto diag_step = [&](int J, bool transposed, int buf) {
#pragma unroll
        for (int r = 0; r < R; ++r) sh.sb[w][lane][r] = f[r];
        __syncwarp();
        float x[R];
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = 0.0f;
#pragma unroll 8
        for (int k = 0; k < 32; ++k) {
            const float l = transposed ? sh.inv[J][k][lane] : sh.inv[J][lane][k];
#pragma unroll
            for (int r = 0; r < R; ++r) x[r] = fmaf(l, sh.sb[w][k][r], x[r]);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            f[r] = x[r];
            sh.sx[buf][lane][r] = x[r];
        }
    };
    // forward: L y = b, blocks ascending; rows below take L(i, block) * y_block
    for (int J = 0; J < nblk; ++J) {
        const int j0 = J * 32, buf = J & 1;
        float lv[32];
        const bool below = (w > J && t < n);
        if (below) {
#pragma unroll
            for (int k = 0; k < 32; ++k) lv[k] = (j0 + k < n) ? SA[t + (size_t)(j0 + k) * n] : 0.0f;
        }
        if (w == J) diag_step(J, false, buf);
        __syncthreads();
        if (below) {
#pragma unroll
            for (int k = 0; k < 32; ++k) {
#pragma unroll
                for (int r = 0; r < R; ++r) f[r] = fmaf(-lv[k], sh.sx[buf][k][r], f[r]);
            }
        }
    }
    // backward: L^T x = y, blocks descending; rows above take L(block, i)^T * x_block
    for (int J = nblk - 1; J >= 0; --J) {
        const int j0 = J * 32, buf = (2 * nblk - 1 - J) & 1;
        float uv[32];
        const bool above = (w < J);
        if (above) {
#pragma unroll
            for (int k = 0; k < 32; ++k) uv[k] = (j0 + k < n) ? SA[j0 + k + (size_t)t * n] : 0.0f;
        }
        if (w == J) diag_step(J, true, buf);
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

template <int NT, int R>
__global__ void __launch_bounds__(NT, (NT >= 512 ? 1 : 512 / NT))
dsposv_refine_vkernel(WorkList wl, const int* n_arr, const int* nrhs_arr, double** dA_array, const int* ldda,
                      double** dB_array, const int* lddb, double** dX_array, const int* lddx, float** dS_array,
                      CholMixedWs ws, int* iter_array) {
    extern __shared__ __align__(16) unsigned char chol_refine_smem[];
    CholRefineSmem<NT, R>& sh = *reinterpret_cast<CholRefineSmem<NT, R>*>(chol_refine_smem);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (int it = blockIdx.x; it < wl.size(); it += gridDim.x) {
        const int id = wl.at(it);
        if (iter_array[id] < 0) continue;        // conversion already failed (block-uniform)
        const int n = n_arr[id], nrhs = nrhs_arr[id];
        if (ws.sinfo[id] != 0) {                 // not positive definite in single precision
            if (t == 0) { iter_array[id] = -3; ws.fkey[id] = n; }
            continue;
        }
        const double* A = dA_array[id];
        const double* B = dB_array[id];
        double* X = dX_array[id];
        const int lda = ldda[id], ldb = lddb[id], ldx = lddx[id];
        const float* SA = dS_array[id];
        const double cte = ws.anrm[id] * (DBL_EPSILON * 0.5) * sqrt((double)n);
        const int nblk = (n + 31) / 32;
        for (int J = w; J < nblk; J += NT / 32) chol_invert_diag_block<NT, R>(SA, n, J, lane, sh);
        __syncthreads();
        int iter_out = 0;
        for (int c0 = 0; c0 < nrhs && iter_out >= 0; c0 += R) {
            double b[R], x[R], res[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                b[r] = (t < n && c0 + r < nrhs) ? B[t + (size_t)(c0 + r) * ldb] : 0.0;
                x[r] = 0.0;
                res[r] = b[r];
            }
            int iiter = 0, stalls = 0;
            double prev_ratio = 1e300;
            for (;;) {
                bool ovf = false;
                float f[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    ovf |= !(fabs(res[r]) <= (double)FLT_MAX);
                    f[r] = (float)res[r];
                }
                if (__syncthreads_or(ovf)) { iter_out = -2; break; }
                chol_refine_solve<NT, R>(SA, n, f, sh);
                if (t < n) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        x[r] += (double)f[r];
                        sh.xs[t][r] = x[r];
                    }
                }
                __syncthreads();
                // R = B - A X with A symmetric, lower triangle stored
#pragma unroll
                for (int r = 0; r < R; ++r) res[r] = b[r];
                if (t < n) {
#pragma unroll 8
                    for (int j = 0; j <= t; ++j) {
                        const double a = A[t + (size_t)j * lda];
#pragma unroll
                        for (int r = 0; r < R; ++r) res[r] = fma(-a, sh.xs[j][r], res[r]);
                    }
#pragma unroll 8
                    for (int j = t + 1; j < n; ++j) {
                        const double a = A[j + (size_t)t * lda];
#pragma unroll
                        for (int r = 0; r < R; ++r) res[r] = fma(-a, sh.xs[j][r], res[r]);
                    }
                }
                double xn[R], rn[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    xn[r] = (t < n && c0 + r < nrhs) ? fabs(x[r]) : 0.0;
                    rn[r] = (t < n && c0 + r < nrhs) ? fabs(res[r]) : 0.0;
                }
                // block-wide maxima per right-hand side
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    for (int off = 16; off > 0; off >>= 1) {
                        xn[r] = fmax(xn[r], __shfl_xor_sync(kFullMask, xn[r], off));
                        rn[r] = fmax(rn[r], __shfl_xor_sync(kFullMask, rn[r], off));
                    }
                }
                __syncthreads();
                if (lane == 0) {
#pragma unroll
                    for (int r = 0; r < R; ++r) { sh.red[0][w][r] = xn[r]; sh.red[1][w][r] = rn[r]; }
                }
                __syncthreads();
                bool ok = true;
                double ratio = 0.0;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    double xm = 0.0, rm = 0.0;
                    for (int k = 0; k < NT / 32; ++k) { xm = fmax(xm, sh.red[0][k][r]); rm = fmax(rm, sh.red[1][k][r]); }
                    if (c0 + r < nrhs) {
                        ok &= (rm <= xm * cte);
                        ratio = fmax(ratio, rm / fmax(xm * cte, DBL_MIN));
                    }
                }
                if (ok) break;
                ++iiter;
                stalls = (ratio > 0.5 * prev_ratio) ? stalls + 1 : 0;
                prev_ratio = ratio;
                if (iiter >= kCholItermax || stalls >= 2) { iter_out = -kCholItermax - 1; break; }
            }
            if (iter_out < 0) break;
            iter_out = max(iter_out, iiter);
            if (t < n) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (c0 + r < nrhs) X[t + (size_t)(c0 + r) * ldx] = x[r];
            }
            __syncthreads();
        }
        if (t == 0) {
            iter_array[id] = iter_out;
            ws.fkey[id] = iter_out < 0 ? n : 0;
        }
        __syncthreads();
    }
}

// ---- 3. fallback helper: X = B for the listed instances ----
__global__ void copy_rhs_vkernel(WorkList wl, const int* n_arr, const int* nrhs_arr, double** dB_array,
                                 const int* lddb, double** dX_array, const int* lddx) {
    for (int it = blockIdx.x; it < wl.size(); it += gridDim.x) {
        const int id = wl.at(it);
        const int n = n_arr[id], nrhs = nrhs_arr[id], ldb = lddb[id], ldx = lddx[id];
        const double* B = dB_array[id];
        double* X = dX_array[id];
        for (int idx = threadIdx.x; idx < n * nrhs; idx += blockDim.x) {
            const int i = idx % n, c = idx / n;
            X[i + (size_t)c * ldx] = B[i + (size_t)c * ldb];
        }
    }
}

// X = B for every instance with fkey set: each warp scans 32 instances with a ballot
// and copies the flagged ones together (the fallback is rare, so most warps copy nothing).
__global__ void copy_rhs_flagged_kernel(const int* fkey, int batch, const int* n_arr, const int* nrhs_arr,
                                        double** dB_array, const int* lddb, double** dX_array, const int* lddx) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int c0 = gw * 32; c0 < batch; c0 += nw * 32) {
        const int i = c0 + lane;
        unsigned m = __ballot_sync(0xffffffffu, i < batch && fkey[i] != 0);
        while (m) {
            const int id = c0 + __ffs(m) - 1;
            m &= m - 1;
            const int n = n_arr[id], nrhs = nrhs_arr[id], ldb = lddb[id], ldx = lddx[id];
            const double* B = dB_array[id];
            double* X = dX_array[id];
            for (int idx = lane; idx < n * nrhs; idx += 32) {
                const int r = idx % n, c = idx / n;
                X[r + (size_t)c * ldx] = B[r + (size_t)c * ldb];
            }
        }
    }
}

// ---- host driver ----
static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <typename K>
static int persistent_grid(K kernel, int threads, size_t smem, int bound) {
    return std::max(1, std::min(bound, resident_blocks((const void*)kernel, threads, smem)));
}

template <int NT>
static void launch_bucket_stage(int stage, const WorkList& wl, int batch, const int* n, const int* nrhs, double** A,
                                const int* lda, double** B, const int* ldb, double** X, const int* ldx, float** S,
                                const CholMixedWs& ws, int* iter, cudaStream_t s) {
    constexpr int R = 4;
    if (stage == 0) {
        auto k = dlat2s_norm_vkernel<NT>;
        k<<<persistent_grid(k, NT, 0, batch), NT, 0, s>>>(wl, n, A, lda, S, ws, iter);
    } else {
        auto k = dsposv_refine_vkernel<NT, R>;
        const int smem = (int)sizeof(CholRefineSmem<NT, R>);
        ensure_dynamic_smem((const void*)k, smem);
        k<<<persistent_grid(k, NT, smem, batch), NT, smem, s>>>(wl, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter);
    }
}

static void bucket_stage(int edge, int stage, const WorkList& wl, int batch, const int* n, const int* nrhs,
                         double** A, const int* lda, double** B, const int* ldb, double** X, const int* ldx,
                         float** S, const CholMixedWs& ws, int* iter, cudaStream_t s) {
    if (edge <= 32) launch_bucket_stage<32>(stage, wl, batch, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter, s);
    else if (edge <= 64) launch_bucket_stage<64>(stage, wl, batch, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter, s);
    else if (edge <= 128) launch_bucket_stage<128>(stage, wl, batch, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter, s);
    else if (edge <= 256) launch_bucket_stage<256>(stage, wl, batch, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter, s);
    else launch_bucket_stage<512>(stage, wl, batch, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter, s);
}

bool dsposv_vbatched_supported(int max_n) { return max_n <= 512; }

magma_int_t dsposv_var(const int* n, const int* nrhs, double** A, const int* lda, double** B, const int* ldb,
                       double** X, const int* ldx, float** S, int* iter, int* info, int batch, int max_n,
                       int max_nrhs, magma_queue_t queue) {
    const int top = chol_bucket_of(max_n);
    if (top < 0 || !dsposv_vbatched_supported(max_n)) return MAGMA_ERR_NOT_SUPPORTED;
    const size_t bw = sizeof(int) * bucketize_ws_ints(batch, kCholBuckets);
    const size_t bytes = align256(sizeof(int) * batch) + align256(sizeof(double) * batch) +
                         2 * align256(sizeof(int) * (batch + 1)) + 2 * align256(bw);
    char* p = static_cast<char*>(queue_workspace(queue, bytes));
    if (!p) return MAGMA_ERR_DEVICE_ALLOC;
    CholMixedWs ws;
    ws.sinfo = reinterpret_cast<int*>(p);   p += align256(sizeof(int) * batch);
    ws.anrm = reinterpret_cast<double*>(p); p += align256(sizeof(double) * batch);
    ws.fkey = reinterpret_cast<int*>(p);    p += align256(sizeof(int) * (batch + 1));
    ws.ldsa = reinterpret_cast<int*>(p);    p += align256(sizeof(int) * (batch + 1));
    int* bws_n = reinterpret_cast<int*>(p); p += align256(bw);
    int* bws_f = reinterpret_cast<int*>(p);
    cudaStream_t s = queue->stream;
    cudaMemsetAsync(info, 0, sizeof(int) * batch, s);
    cudaMemsetAsync(iter, 0, sizeof(int) * batch, s);
    cudaMemsetAsync(ws.fkey, 0, sizeof(int) * batch, s);   // n = 0 instances never need the fallback
    int *counts, *lists;
    magma_int_t rc = bucketize(n, batch, kCholEdges, kCholBuckets, s, bws_n, &counts, &lists);
    if (rc) return rc;
    const LuSizes sz32{0, 0, 0, 0, 0, n, n, ws.ldsa, nullptr, nullptr};
    // buckets are independent: each bucket's three stages run in order on its own auxiliary stream
    if ((rc = queue_fork(queue))) return rc;
    for (int b = top; b >= 0; --b) {
        cudaStream_t sb = queue_aux(queue, top - b);
        const WorkList wl{lists + (size_t)b * batch, counts + b, 0};
        bucket_stage(kCholEdges[b], 0, wl, batch, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter, sb);
        chol_bucket<float>(b, wl, batch, true, sz32, false, S, nullptr, ws.sinfo, true, false, 0, sb);
        bucket_stage(kCholEdges[b], 1, wl, batch, n, nrhs, A, lda, B, ldb, X, ldx, S, ws, iter, sb);
    }
    queue_join(queue);
    if ((rc = launch_status())) return rc;
    // FP64 fallback for the instances that set fkey: X = B, then dpotrf + dpotrs on A, X
    rc = bucketize(ws.fkey, batch, kCholEdges, kCholBuckets, s, bws_f, &counts, &lists);
    if (rc) return rc;
    const LuSizes sz64{0, 0, 0, 0, 0, n, n, lda, ldx, nrhs};
    if (tuning().chol_queue && top < kCholBuckets - 1) {
        // one copy and one persistent factor + solve launch over every size
        copy_rhs_flagged_kernel<<<std::max(1, std::min(ceildiv(batch, 256), 1184)), 256, 0, s>>>(
            ws.fkey, batch, n, nrhs, B, ldb, X, ldx);
        chol_queue<double>(counts, lists, batch, top, counts + kCholBuckets, sz64, false, A, X, info, true, true,
                           max_nrhs, s);
        return launch_status();
    }
    if ((rc = queue_fork(queue))) return rc;
    for (int b = top; b >= 0; --b) {
        cudaStream_t sb = queue_aux(queue, top - b);
        const WorkList wl{lists + (size_t)b * batch, counts + b, 0};
        copy_rhs_vkernel<<<std::min(batch, 1184), 256, 0, sb>>>(wl, n, nrhs, B, ldb, X, ldx);
        chol_bucket<double>(b, wl, batch, true, sz64, false, A, X, info, true, true, max_nrhs, sb);
    }
    queue_join(queue);
    return launch_status();
}

}  // namespace mb200

using namespace mb200;

extern "C" {

magma_int_t magma_dsposv_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs,
                                              double** dA_array, magma_int_t* ldda, double** dB_array,
                                              magma_int_t* lddb, double** dX_array, magma_int_t* lddx,
                                              float** dworks_array, magma_int_t* iter_array,
                                              magma_int_t* info_array, magma_int_t batchCount, magma_int_t max_n,
                                              magma_int_t max_nrhs, magma_queue_t queue) {
    if (uplo != MagmaLower) return MAGMA_ERR_NOT_SUPPORTED;   // as magma_dpotrf_vbatched's lower-only kernels
    if (batchCount <= 0) return 0;
    if (max_n <= 0 || max_nrhs <= 0) {
        cudaMemsetAsync(info_array, 0, sizeof(int) * batchCount, queue->stream);
        cudaMemsetAsync(iter_array, 0, sizeof(int) * batchCount, queue->stream);
        return 0;
    }
    return dsposv_var(n, nrhs, dA_array, ldda, dB_array, lddb, dX_array, lddx, dworks_array, iter_array,
                      info_array, batchCount, max_n, max_nrhs, queue);
}

// Checks: uplo -1, n -2, nrhs -3, ldda < n -5, lddb < n -7, lddx < n -9, batchCount -13
// (magma_dsposv_gpu's argument order with per-instance arrays).
magma_int_t magma_dsposv_vbatched(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                  magma_int_t* ldda, double** dB_array, magma_int_t* lddb, double** dX_array,
                                  magma_int_t* lddx, float** dworks_array, magma_int_t* iter_array,
                                  magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue) {
    magma_int_t arginfo = 0;
    int r[6] = {0, 0, 0, 0, 0, 0};
    if (uplo != MagmaLower && uplo != MagmaUpper) arginfo = -1;
    else if (batchCount < 0) arginfo = -13;
    else if (batchCount > 0) {
        magma_int_t rc = reduce_sizes(n, nrhs, nullptr, batchCount, queue, r);
        if (rc) return rc;
        if (r[3] < 0) arginfo = -2;
        else if (r[4] < 0) arginfo = -3;
        int sa = 0;
        if (!arginfo && (rc = ld_slack(n, ldda, batchCount, queue, &sa)) != 0) return rc;
        if (!arginfo && sa < 0) arginfo = -5;
        if (!arginfo && (rc = ld_slack(n, lddb, batchCount, queue, &sa)) != 0) return rc;
        if (!arginfo && sa < 0) arginfo = -7;
        if (!arginfo && (rc = ld_slack(n, lddx, batchCount, queue, &sa)) != 0) return rc;
        if (!arginfo && sa < 0) arginfo = -9;
    }
    if (arginfo != 0) {
        magma_xerbla(__func__, -arginfo);
        return arginfo;
    }
    return magma_dsposv_vbatched_max_nocheck(uplo, n, nrhs, dA_array, ldda, dB_array, lddb, dX_array, lddx,
                                             dworks_array, iter_array, info_array, batchCount, r[0], r[1], queue);
}

}  // extern "C"
