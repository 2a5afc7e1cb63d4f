// mixed.cu -- batched mixed-precision LU solve: FP32 factorisation, FP64
// iterative refinement, FP64 fallback (magma_dsgesv_batched).
//
// Per instance this follows magma_dsgesv_gpu (src/zcgesv_gpu.cpp:144-365):
//   Anrm = ||A||_inf, cte = Anrm * eps * sqrt(n)            (:208-209, BWDMAX = 1)
//   SA = single(A); overflow -> iter = -2, fallback          (:220-224)
//   SA = L U in single; info > 0 -> iter = -3, fallback      (:227-231)
//   X = SA^-1 B; R = B - A X (double); done if every RHS j has
//       max|R_j| <= max|X_j| * cte                           (:251-281) -> iter = 0
//   loop iiter = 1 .. ITERMAX-1: C = SA^-1 R; X += C; R = B - A X; test  (:284-350)
//   no convergence -> iter = -ITERMAX-1 = -31, fallback      (:351-360)
//   fallback: dgetrf(A) + dgetrs (A overwritten, ipiv the double pivots)
// Additionally refinement stops early (iter = -31) when the residual ratio
// fails to halve over two consecutive iterations, so an instance that cannot
// converge does not spend 29 iterations before its fallback.
//
// Unlike the reference there is no host synchronisation: every instance runs
// its own refinement loop inside one kernel launch, and the instances that
// need the fallback are collected into a device list that the FP64 kernels
// walk. Single-precision pivots are returned in ipiv when iter >= 0 (LAPACK
// dsgesv convention).
#include "internal.h"
#include "batched_kernels.h"
#include "getrs_blocked.cuh"
#include "mixed_refine.cuh"
#include "lu_tc.h"
#include "tuning.h"
#include "lu_sizes.h"
#include "vbatched.h"
#include <cfloat>

namespace mb200 {

constexpr int kItermax = 30;

// Workspace of one call, carved from the queue workspace.
struct MixedWs {
    float* SA;          // batch * n * n floats
    float** SA_ptr;     // batch
    int* sinfo;         // batch
    double* anrm;       // batch
    float* R;           // batch * n * R floats (single-precision right-hand sides)
    int* fail_count;    // 1
    int* fail_list;     // batch
    int* err;           // 1: a tensor-core wait timed out (the instances went to the fallback)
};

static size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

static size_t mixed_ws_bytes(int n, int batch, int R) {
    return align_up(sizeof(float) * (size_t)batch * n * n) + align_up(sizeof(float*) * batch) +
           align_up(sizeof(int) * batch) + align_up(sizeof(double) * batch) +
           align_up(sizeof(float) * (size_t)batch * n * R) + align_up(sizeof(int)) + align_up(sizeof(int) * batch) +
           align_up(sizeof(int));
}

static MixedWs carve(void* base, int n, int batch, int R) {
    char* p = static_cast<char*>(base);
    MixedWs w;
    w.SA = reinterpret_cast<float*>(p);       p += align_up(sizeof(float) * (size_t)batch * n * n);
    w.SA_ptr = reinterpret_cast<float**>(p);  p += align_up(sizeof(float*) * batch);
    w.sinfo = reinterpret_cast<int*>(p);      p += align_up(sizeof(int) * batch);
    w.anrm = reinterpret_cast<double*>(p);    p += align_up(sizeof(double) * batch);
    w.R = reinterpret_cast<float*>(p);        p += align_up(sizeof(float) * (size_t)batch * n * R);
    w.fail_count = reinterpret_cast<int*>(p); p += align_up(sizeof(int));
    w.fail_list = reinterpret_cast<int*>(p);  p += align_up(sizeof(int) * batch);
    w.err = reinterpret_cast<int*>(p);
    return w;
}

__device__ __forceinline__ void push_fail(int id, int* fail_count, int* fail_list) {
    const int slot = atomicAdd(fail_count, 1);
    fail_list[slot] = id;
}

// ---- 1. SA = single(A), ||A||_inf, overflow check. One block per instance. ----
template <int NT>
__global__ void __launch_bounds__(NT)
dlag2s_norm_kernel(int n, double** dA_array, int lda, MixedWs ws, int* iter_array) {
    const int id = blockIdx.x;
    const double* A = dA_array[id];
    float* SA = ws.SA + (size_t)id * n * n;
    if (threadIdx.x == 0) ws.SA_ptr[id] = SA;
    __shared__ double red[NT / 32];
    __shared__ int ovf;
    if (threadIdx.x == 0) ovf = 0;
    __syncthreads();
    double rowsum_max = 0.0;
    bool overflow = false;
    for (int i = threadIdx.x; i < n; i += NT) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) {
            const double a = A[i + (size_t)j * lda];
            s += fabs(a);
            overflow |= !(fabs(a) <= (double)FLT_MAX);   // also catches NaN
            SA[i + (size_t)j * n] = (float)a;
        }
        rowsum_max = fmax(rowsum_max, s);
    }
    for (int off = 16; off > 0; off >>= 1) rowsum_max = fmax(rowsum_max, __shfl_xor_sync(kFullMask, rowsum_max, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rowsum_max;
    if (overflow) ovf = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < NT / 32; ++w) m = fmax(m, red[w]);
        ws.anrm[id] = m;
        if (ovf) {
            iter_array[id] = -2;
            push_fail(id, ws.fail_count, ws.fail_list);
        }
    }
}

// ---- 2. refinement, one block per instance, thread = row (mixed_refine.cuh) ----
template <int NT, int R>
__global__ void __launch_bounds__(NT, (NT >= 512 ? 1 : 512 / NT))
dsgesv_refine_kernel(int n, int nrhs, double** dA_array, int lda, int** ipiv_array, double** dB_array, int ldb,
                     double** dX_array, int ldx, MixedWs ws, int* iter_array) {
    extern __shared__ __align__(16) unsigned char refine_smem[];
    RefineSmem<NT, R>& sh = *reinterpret_cast<RefineSmem<NT, R>*>(refine_smem);
    const int id = blockIdx.x;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (iter_array[id] < 0) return;          // conversion already failed
    if (ws.sinfo[id] != 0) {                 // singular in single precision
        if (t == 0) {
            iter_array[id] = -3;
            push_fail(id, ws.fail_count, ws.fail_list);
        }
        return;
    }
    const double* A = dA_array[id];
    const double* B = dB_array[id];
    double* X = dX_array[id];
    const float* SA = ws.SA + (size_t)id * n * n;
    const int* ipiv = ipiv_array[id];
    const double cte = ws.anrm[id] * (DBL_EPSILON * 0.5) * sqrt((double)n);
    for (int k = t; k < n; k += NT) sh.ipiv[k] = ipiv[k];
    const int nblk = (n + 31) / 32;
    for (int J = w; J < nblk; J += NT / 32) invert_diag_block<NT, R>(SA, n, J, lane, sh);
    __syncthreads();
    const int fwd = (t < n) ? laswp_target(sh.ipiv, n, t, false) : t;
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
            // column t of A to L2 while the solve below runs, for this pass's residual
            if (t < n) prefetch_l2(A + (size_t)t * lda, (unsigned)n * 8u);
            // C = SA^-1 res in single precision (res = B on the first pass)
            bool ovf = false;
            float f[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                ovf |= !(fabs(res[r]) <= (double)FLT_MAX);
                f[r] = (float)res[r];
            }
            if (__syncthreads_or(ovf)) { iter_out = -2; break; }
            if (t < n) {
#pragma unroll
                for (int r = 0; r < R; ++r) sh.xch[fwd][r] = f[r];
            }
            __syncthreads();
#pragma unroll
            for (int r = 0; r < R; ++r) f[r] = (t < n) ? sh.xch[t][r] : 0.0f;
            refine_solve<NT, R>(SA, n, f, sh);
            if (t < n) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    x[r] += (double)f[r];
                    sh.xs[t][r] = x[r];
                }
            }
            __syncthreads();
            // R = B - A X in double precision
#pragma unroll
            for (int r = 0; r < R; ++r) res[r] = b[r];
            if (t < n) {
#pragma unroll(NT >= 256 ? 32 : 16)
                for (int j = 0; j < n; ++j) {
                    const double a = A[t + (size_t)j * lda];
#pragma unroll
                    for (int r = 0; r < R; ++r) res[r] = fma(-a, sh.xs[j][r], res[r]);
                }
            }
            // max |X_j| and max |R_j| per right-hand side
            double xn[R], rn[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                xn[r] = (t < n && c0 + r < nrhs) ? fabs(x[r]) : 0.0;
                rn[r] = (t < n && c0 + r < nrhs) ? fabs(res[r]) : 0.0;
            }
            refine_max2<NT, R>(xn, rn, sh);
            bool ok = true;
            double ratio = 0.0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (c0 + r < nrhs) {
                    ok &= (rn[r] <= xn[r] * cte);
                    ratio = fmax(ratio, rn[r] / fmax(xn[r] * cte, DBL_MIN));
                }
            }
            if (ok) break;
            ++iiter;
            stalls = (ratio > 0.5 * prev_ratio) ? stalls + 1 : 0;
            prev_ratio = ratio;
            if (iiter >= kItermax || stalls >= 2) { iter_out = -kItermax - 1; break; }
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
        if (iter_out < 0) push_fail(id, ws.fail_count, ws.fail_list);
    }
}

// ---- 3. fallback helper: X = B for the listed instances ----
__global__ void copy_rhs_kernel(WorkList wl, int n, int nrhs, double** dB_array, int ldb, double** dX_array, int ldx) {
    for (int w = blockIdx.x; w < wl.size(); w += gridDim.x) {
        const int id = wl.at(w);
        const double* B = dB_array[id];
        double* X = dX_array[id];
        for (int idx = threadIdx.x; idx < n * nrhs; idx += blockDim.x) {
            const int i = idx % n, c = idx / n;
            X[i + (size_t)c * ldx] = B[i + (size_t)c * ldb];
        }
    }
}

template <int NT, int R>
static void launch_refine(int n, int nrhs, double** A, int lda, int** ipiv, double** B, int ldb, double** X, int ldx,
                          const MixedWs& w, int* iter, int batch, cudaStream_t s) {
    auto k = dsgesv_refine_kernel<NT, R>;
    const int smem = (int)sizeof(RefineSmem<NT, R>);
    ensure_dynamic_smem((const void*)k, smem);
    k<<<batch, NT, smem, s>>>(n, nrhs, A, lda, ipiv, B, ldb, X, ldx, w, iter);
}

bool dsgesv_supported(int n) { return n <= 512; }

// The tensor-core LU serves n = 96..256 in steps of 32 (smaller orders use the
// register kernels) unless the tuning table turns it off, as a whole (it starts from
// MAGMA_B200_TENSOR_CORE_LU=0 in the environment) or per order (magma_b200_autotune
// measures both paths at each order).
static bool use_tensor_core_lu(int n) {
    return tuning().mixed_tc_lu && n > 64 && lu_tc_supported(n) && tuning().mixed_tc_n[(n - 96) / 32];
}

magma_int_t dsgesv_batched(int n, int nrhs, double** dA, int lda, int** ipiv, double** dB, int ldb, double** dX,
                           int ldx, int* iter, int* info, int batch, magma_queue_t queue) {
    constexpr int R = 4;
    if (!dsgesv_supported(n)) return MAGMA_ERR_NOT_SUPPORTED;
    cudaStream_t s = queue->stream;
    void* base = queue_workspace(queue, mixed_ws_bytes(n, batch, R));
    if (!base) return MAGMA_ERR_DEVICE_ALLOC;
    MixedWs w = carve(base, n, batch, R);
    cudaMemsetAsync(info, 0, sizeof(int) * batch, s);
    cudaMemsetAsync(iter, 0, sizeof(int) * batch, s);
    cudaMemsetAsync(w.fail_count, 0, sizeof(int), s);
    magma_int_t rc = 0;
    queue_stage_begin(queue);   // stages: LU, refinement, FP64 fallback
    const bool tc = use_tensor_core_lu(n);
    if (tc) {
        // 1-3. conversion, norm, an FP32-accurate LU on the tensor cores (TMEM-resident)
        // and the FP64 refinement, each instance in one block
        cudaMemsetAsync(w.err, 0, sizeof(int), s);
        const TcLuArgs args{n,  batch, lda, dA, w.SA, ipiv, w.sinfo, w.anrm, iter, w.fail_count, w.fail_list, w.err,
                            0, 1,   // wait bound and MMA issue are set by lu_tc_launch
                            nrhs, dB, ldb, dX, ldx};
        if ((rc = lu_tc_launch(args, s))) return rc;
    } else {
        // 1. conversion + norm
        if (n <= 128) dlag2s_norm_kernel<128><<<batch, 128, 0, s>>>(n, dA, lda, w, iter);
        else dlag2s_norm_kernel<256><<<batch, 256, 0, s>>>(n, dA, lda, w, iter);
        // 2. single-precision LU of SA, pivots straight into the caller's ipiv
        const WorkList all{nullptr, nullptr, batch};
        const LuSizes szs{n, n, n, n, R, nullptr, nullptr, nullptr, nullptr, nullptr};
        rc = small_lu_supported(n, n) ? getrf_small<float>(all, batch, false, szs, n, n, w.SA_ptr, ipiv, w.sinfo, s)
                                      : getrf_blocked<float>(all, batch, false, szs, n, w.SA_ptr, ipiv, w.sinfo, s);
        if (rc) return rc;
    }
    queue_stage_mark(queue);
    // 3. refinement (already done inside the tensor-core kernel)
    if (!tc) {
        if (n <= 64) launch_refine<64, R>(n, nrhs, dA, lda, ipiv, dB, ldb, dX, ldx, w, iter, batch, s);
        else if (n <= 128) launch_refine<128, R>(n, nrhs, dA, lda, ipiv, dB, ldb, dX, ldx, w, iter, batch, s);
        else if (n <= 256) launch_refine<256, R>(n, nrhs, dA, lda, ipiv, dB, ldb, dX, ldx, w, iter, batch, s);
        else launch_refine<512, R>(n, nrhs, dA, lda, ipiv, dB, ldb, dX, ldx, w, iter, batch, s);
        if ((rc = launch_status())) return rc;
    }
    queue_stage_mark(queue);
    // 4. FP64 fallback on the listed instances (the list length stays on the device)
    const WorkList failed{w.fail_list, w.fail_count, 0};
    const LuSizes szd{n, n, lda, ldx, nrhs, nullptr, nullptr, nullptr, nullptr, nullptr};
    rc = small_lu_supported(n, n) ? getrf_small<double>(failed, batch, true, szd, n, n, dA, ipiv, info, s)
                                  : getrf_blocked<double>(failed, batch, true, szd, n, dA, ipiv, info, s);
    if (rc) return rc;
    copy_rhs_kernel<<<std::min(batch, 1184), 256, 0, s>>>(failed, n, nrhs, dB, ldb, dX, ldx);
    rc = small_lu_supported(n, n) ? getrs_small<double>(failed, batch, true, false, szd, n, nrhs, dA, ipiv, dX, s)
                                  : getrs_blocked<double>(failed, batch, true, false, szd, n, nrhs, dA, ipiv, dX, s);
    queue_stage_mark(queue);
    return rc ? rc : launch_status();
}

}  // namespace mb200
