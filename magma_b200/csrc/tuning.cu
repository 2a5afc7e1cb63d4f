// tuning.cu -- kernel-variant table and its autotuner.
//
// The dispatchers of the variable-size GEMM (tile shape per size bucket), of
// the mixed-precision solve (tensor-core or CUDA-core FP32 LU) and of the FP64
// blocked LU (trailing update on the tensor cores or the FP64 pipe, per size
// bucket) read one process-wide table. Defaults are built in; MAGMA_B200_TUNING=<file> loads a
// saved table at first use; magma_b200_autotune() measures every variant on the
// queue's device with synthetic problems of each bucket and keeps the fastest.
// Every variant of a family computes bit-identical results (same fma order per
// output element), so tuning changes speed only; the one exception is the FP32 GEMM
// tile on the tcgen05 tensor cores (split TF32), held to the reference tester's bound.
#include "internal.h"
#include "tuning.h"
#include "../../include/magma_b200.h"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <vector>

namespace mb200 {

static TuningTable g_table;
static std::once_flag g_once;

// Built-in defaults: what magma_b200_autotune picked on B200s, with the GEMM tiles
// checked on the C2 workload (20,000 instances, M, N, K in 8..128): FP64 16x16 / 32x32
// CUDA-core tiles up to max(M, N) = 32 and the DMMA tile above (7.38 TF/s, against 6.94
// with CUDA-core tiles throughout); FP32 CUDA-core tiles up to 64 and the tcgen05 tile
// above (14.6 TF/s, against 10.7).
static void set_defaults(TuningTable& t) {
    const int gemm[2][kGemmBuckets] = {{2, 1, 3, 3}, {2, 1, 1, 3}};
    for (int p = 0; p < 2; ++p)
        for (int b = 0; b < kGemmBuckets; ++b) t.gemm_variant[p][b] = gemm[p][b];
    const char* e = std::getenv("MAGMA_B200_TENSOR_CORE_LU");
    t.mixed_tc_lu = (e && e[0] == '0') ? 0 : 1;
    // the FP64 pipe's update in every bucket (DMMA is slower at each size: n = 256
    // 684 against 734 us in ncu, 1,024 within noise)
    for (int b = 0; b < kLuBlockedBuckets; ++b) t.lu_dmma[b] = 0;
    // tensor-core LU from n = 160 on; the CUDA-core FP32 LU is faster at n = 96 and 128
    for (int i = 0; i < kMixedTcOrders; ++i) t.mixed_tc_n[i] = (i >= 2);
    t.chol_queue = 1;   // one launch for the variable-size Cholesky
    t.lu_queue = 0;     // one launch per size bucket for the variable-size LU
}

static void to_values(const TuningTable& t, int* v) {
    int i = 0;
    for (int p = 0; p < 2; ++p)
        for (int b = 0; b < kGemmBuckets; ++b) v[i++] = t.gemm_variant[p][b];
    v[i++] = t.mixed_tc_lu;
    for (int b = 0; b < kLuBlockedBuckets; ++b) v[i++] = t.lu_dmma[b];
    for (int k = 0; k < kMixedTcOrders; ++k) v[i++] = t.mixed_tc_n[k];
    v[i++] = t.chol_queue;
    v[i++] = t.lu_queue;
}

// count kTuningValues, or kTuningValuesV1 / V2 / V3 / V4 (tables saved before the later
// entries existed: those keep their current values).
static bool from_values(const int* v, int count, TuningTable& t) {
    if (count != kTuningValues && count != kTuningValuesV1 && count != kTuningValuesV2 &&
        count != kTuningValuesV3 && count != kTuningValuesV4)
        return false;
    for (int i = 0; i < 2 * kGemmBuckets; ++i)
        if (v[i] < 0 || v[i] > 3) return false;   // 3: the tensor-core tile (FP64 DMMA, FP32 tcgen05)
    for (int i = 2 * kGemmBuckets; i < count; ++i)
        if (v[i] != 0 && v[i] != 1) return false;
    int i = 0;
    for (int p = 0; p < 2; ++p)
        for (int b = 0; b < kGemmBuckets; ++b) t.gemm_variant[p][b] = v[i++];
    t.mixed_tc_lu = v[i++];
    if (count >= kTuningValuesV2)
        for (int b = 0; b < kLuBlockedBuckets; ++b) t.lu_dmma[b] = v[i++];
    if (count >= kTuningValuesV3)
        for (int k = 0; k < kMixedTcOrders; ++k) t.mixed_tc_n[k] = v[i++];
    if (count >= kTuningValuesV4) t.chol_queue = v[i++];
    if (count >= kTuningValues) t.lu_queue = v[i++];
    return true;
}

static bool load_file(const char* path, TuningTable& t) {
    FILE* f = std::fopen(path, "r");
    if (!f) return false;
    char magic[64] = {0};
    int v[kTuningValues];
    bool ok = std::fscanf(f, "%63s", magic) == 1;
    const int count = !ok ? 0 : std::strcmp(magic, "magma_b200_tuning_v5") == 0 ? kTuningValues
                             : std::strcmp(magic, "magma_b200_tuning_v4") == 0 ? kTuningValuesV4
                             : std::strcmp(magic, "magma_b200_tuning_v3") == 0 ? kTuningValuesV3
                             : std::strcmp(magic, "magma_b200_tuning_v2") == 0 ? kTuningValuesV2
                             : std::strcmp(magic, "magma_b200_tuning_v1") == 0 ? kTuningValuesV1 : 0;
    ok = ok && count > 0;
    for (int i = 0; ok && i < count; ++i) ok = std::fscanf(f, "%d", &v[i]) == 1;
    std::fclose(f);
    return ok && from_values(v, count, t);
}

static void init_once() {
    std::call_once(g_once, [] {
        set_defaults(g_table);
        const char* path = std::getenv("MAGMA_B200_TUNING");
        if (path && *path) {
            TuningTable t = g_table;
            if (load_file(path, t)) g_table = t;
            else std::fprintf(stderr, "libmagma_b200: could not read tuning file %s; using defaults\n", path);
        }
    });
}

const TuningTable& tuning() {
    init_once();
    return g_table;
}
TuningTable& tuning_mut() {
    init_once();
    return g_table;
}

}  // namespace mb200

namespace mb200 {

// Deterministic uniform[-1,1) fill (splitmix64 of the index) for the synthetic problems.
template <typename T>
__global__ void tune_fill_kernel(T* x, size_t count, unsigned long long seed) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        x[i] = T(double(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
    }
}

// Adds `shift` to the diagonal of each n x n matrix (keeps the LU benchmark well conditioned).
__global__ void tune_shift_diag_kernel(double* A, int n, int batch, double shift) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * batch; i += gridDim.x * blockDim.x) {
        const int b = i / n, d = i % n;
        A[(size_t)b * n * n + d + (size_t)d * n] += shift;
    }
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    bool alloc(size_t bytes) { return cudaMalloc(&p, bytes) == cudaSuccess; }
};

static float time_ms(cudaStream_t s, const std::function<void()>& fn, int reps) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    fn();   // warm-up (also sizes the queue workspace)
    cudaEventRecord(a, s);
    for (int i = 0; i < reps; ++i) fn();
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
}

// GEMM: for each precision and bucket, 4,096 instances with max(M, N) inside the
// bucket and K ~ U{8..128}; every tile variant is timed through the public
// variable-size entry point with the table pointing the bucket at it.
template <typename T>
static magma_int_t tune_gemm(int prec, magma_queue_t q, unsigned seed) {
    const int count = 4096;
    const int lo[kGemmBuckets] = {1, 17, 33, 65}, hi[kGemmBuckets] = {16, 32, 64, 128};
    for (int b = 0; b < kGemmBuckets; ++b) {
        std::vector<int> M(count + 1), N(count + 1), K(count + 1);
        unsigned long long st = seed * 1000003ull + b;
        auto next = [&](int a, int z) {
            st = st * 6364136223846793005ull + 1442695040888963407ull;
            return a + int((st >> 33) % (unsigned long long)(z - a + 1));
        };
        size_t na = 0, nb = 0, nc = 0;
        std::vector<size_t> oa(count), ob(count), oc(count);
        for (int i = 0; i < count; ++i) {
            M[i] = next(lo[b], hi[b]);
            N[i] = next(lo[b], hi[b]);
            K[i] = next(8, 128);
            oa[i] = na; ob[i] = nb; oc[i] = nc;
            na += (size_t)M[i] * K[i]; nb += (size_t)K[i] * N[i]; nc += (size_t)M[i] * N[i];
        }
        M[count] = N[count] = K[count] = 0;
        DevBuf dA, dB, dC, dP, dI;
        if (!dA.alloc(sizeof(T) * na) || !dB.alloc(sizeof(T) * nb) || !dC.alloc(sizeof(T) * nc) ||
            !dP.alloc(sizeof(T*) * 3 * count) || !dI.alloc(sizeof(int) * 3 * (count + 1)))
            return MAGMA_ERR_DEVICE_ALLOC;
        tune_fill_kernel<T><<<1024, 256, 0, q->stream>>>((T*)dA.p, na, seed + 1);
        tune_fill_kernel<T><<<1024, 256, 0, q->stream>>>((T*)dB.p, nb, seed + 2);
        tune_fill_kernel<T><<<1024, 256, 0, q->stream>>>((T*)dC.p, nc, seed + 3);
        std::vector<T*> ptr(3 * count);
        for (int i = 0; i < count; ++i) {
            ptr[i] = (T*)dA.p + oa[i];
            ptr[count + i] = (T*)dB.p + ob[i];
            ptr[2 * count + i] = (T*)dC.p + oc[i];
        }
        cudaMemcpyAsync(dP.p, ptr.data(), sizeof(T*) * 3 * count, cudaMemcpyHostToDevice, q->stream);
        int* di = (int*)dI.p;
        cudaMemcpyAsync(di, M.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice, q->stream);
        cudaMemcpyAsync(di + count + 1, N.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice, q->stream);
        cudaMemcpyAsync(di + 2 * (count + 1), K.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice, q->stream);
        cudaStreamSynchronize(q->stream);
        int* dm = di; int* dn = di + count + 1; int* dk = di + 2 * (count + 1);
        T** pA = (T**)dP.p; T** pB = pA + count; T** pC = pB + count;
        float best = 1e30f;
        int best_v = tuning().gemm_variant[prec][b];
        for (int v = 0; v < 4; ++v) {
            tuning_mut().gemm_variant[prec][b] = v;
            const float ms = time_ms(q->stream, [&] {
                if (sizeof(T) == 8)
                    magmablas_dgemm_vbatched_max_nocheck(MagmaNoTrans, MagmaNoTrans, dm, dn, dk, 1.0,
                                                         (const double* const*)pA, dm, (const double* const*)pB, dk,
                                                         0.5, (double**)pC, dm, count, hi[b], hi[b], 128, q);
                else
                    magmablas_sgemm_vbatched_max_nocheck(MagmaNoTrans, MagmaNoTrans, dm, dn, dk, 1.0f,
                                                         (const float* const*)pA, dm, (const float* const*)pB, dk,
                                                         0.5f, (float**)pC, dm, count, hi[b], hi[b], 128, q);
            }, 5);
            if (cudaGetLastError() != cudaSuccess) return MAGMA_ERR_UNKNOWN;
            if (ms < best) { best = ms; best_v = v; }
        }
        tuning_mut().gemm_variant[prec][b] = best_v;
    }
    return MAGMA_SUCCESS;
}

// Mixed solve, per order n = 96..256 (step 32): the tensor-core LU with its fused
// refinement against the CUDA-core FP32 LU with the separate refinement kernel, on
// about 128 MB of diagonally dominant systems with 4 right-hand sides each.
static magma_int_t tune_mixed(magma_queue_t q, unsigned seed) {
    const int nrhs = 4;
    for (int o = 0; o < kMixedTcOrders; ++o) {
        const int n = 96 + 32 * o;
        const int batch = std::max(64, (128 << 20) / (8 * n * n));
        DevBuf dA, dA0, dB, dX, dP, dIp, dI;
        const size_t an = (size_t)n * n * batch;
        if (!dA.alloc(8 * an) || !dA0.alloc(8 * an) || !dB.alloc(8 * (size_t)n * nrhs * batch) ||
            !dX.alloc(8 * (size_t)n * nrhs * batch) || !dP.alloc(sizeof(void*) * 4 * batch) ||
            !dIp.alloc(sizeof(int) * (size_t)n * batch) || !dI.alloc(sizeof(int) * 2 * batch))
            return MAGMA_ERR_DEVICE_ALLOC;
        tune_fill_kernel<double><<<1024, 256, 0, q->stream>>>((double*)dA0.p, an, seed + 11 + o);
        tune_shift_diag_kernel<<<256, 256, 0, q->stream>>>((double*)dA0.p, n, batch, 2.0 * n);
        tune_fill_kernel<double><<<1024, 256, 0, q->stream>>>((double*)dB.p, (size_t)n * nrhs * batch, seed + 12 + o);
        std::vector<void*> ptr(4 * batch);
        for (int i = 0; i < batch; ++i) {
            ptr[i] = (double*)dA.p + (size_t)i * n * n;
            ptr[batch + i] = (double*)dB.p + (size_t)i * n * nrhs;
            ptr[2 * batch + i] = (double*)dX.p + (size_t)i * n * nrhs;
            ptr[3 * batch + i] = (int*)dIp.p + (size_t)i * n;
        }
        cudaMemcpyAsync(dP.p, ptr.data(), sizeof(void*) * 4 * batch, cudaMemcpyHostToDevice, q->stream);
        cudaStreamSynchronize(q->stream);
        void** p = (void**)dP.p;
        int* it = (int*)dI.p;
        float best = 1e30f;
        int best_v = tuning().mixed_tc_n[o];
        const int master = tuning().mixed_tc_lu;
        tuning_mut().mixed_tc_lu = 1;
        for (int v = 0; v < 2; ++v) {
            tuning_mut().mixed_tc_n[o] = v;
            const float ms = time_ms(q->stream, [&] {
                cudaMemcpyAsync(dA.p, dA0.p, 8 * an, cudaMemcpyDeviceToDevice, q->stream);
                magma_dsgesv_batched(n, nrhs, (double**)p, n, (int**)(p + 3 * batch), (double**)(p + batch), n,
                                     (double**)(p + 2 * batch), n, it, it + batch, batch, q);
            }, 3);
            if (cudaGetLastError() != cudaSuccess) return MAGMA_ERR_UNKNOWN;
            if (ms < best) { best = ms; best_v = v; }
        }
        tuning_mut().mixed_tc_lu = master;
        tuning_mut().mixed_tc_n[o] = best_v;
    }
    return MAGMA_SUCCESS;
}

// FP64 blocked LU: for each bucket, the two trailing-update variants on a batch of
// about 256 MB of uniform[-1,1] matrices of the bucket's largest order, through
// magma_dgetrf_batched (both variants give bit-identical factors).
static magma_int_t tune_lu_update(magma_queue_t q, unsigned seed) {
    const int orders[kLuBlockedBuckets] = {128, 256, 512, 1024};
    for (int b = 0; b < kLuBlockedBuckets; ++b) {
        const int n = orders[b];
        const int batch = std::max(16, (256 << 20) / (8 * n * n));
        const size_t an = (size_t)n * n * batch;
        DevBuf dA, dA0, dP, dI;
        if (!dA.alloc(8 * an) || !dA0.alloc(8 * an) || !dP.alloc(sizeof(void*) * 2 * batch) ||
            !dI.alloc(sizeof(int) * ((size_t)n * batch + batch)))
            return MAGMA_ERR_DEVICE_ALLOC;
        tune_fill_kernel<double><<<1024, 256, 0, q->stream>>>((double*)dA0.p, an, seed + b);
        std::vector<void*> ptr(2 * batch);
        for (int i = 0; i < batch; ++i) {
            ptr[i] = (double*)dA.p + (size_t)i * n * n;
            ptr[batch + i] = (int*)dI.p + (size_t)i * n;
        }
        cudaMemcpyAsync(dP.p, ptr.data(), sizeof(void*) * 2 * batch, cudaMemcpyHostToDevice, q->stream);
        cudaStreamSynchronize(q->stream);
        void** p = (void**)dP.p;
        int* info = (int*)dI.p + (size_t)n * batch;
        float best = 1e30f;
        int best_v = tuning().lu_dmma[b];
        for (int v = 0; v < 2; ++v) {
            tuning_mut().lu_dmma[b] = v;
            const float ms = time_ms(q->stream, [&] {
                cudaMemcpyAsync(dA.p, dA0.p, 8 * an, cudaMemcpyDeviceToDevice, q->stream);
                magma_dgetrf_batched(n, n, (double**)p, n, (int**)(p + batch), info, batch, q);
            }, 3);
            if (cudaGetLastError() != cudaSuccess) return MAGMA_ERR_UNKNOWN;
            if (ms < best) { best = ms; best_v = v; }
        }
        tuning_mut().lu_dmma[b] = best_v;
    }
    return MAGMA_SUCCESS;
}

// Sets each n x n matrix's diagonal to 2n + its value: with the other lower-triangle
// entries in [-1, 1) the symmetric matrix the lower triangle defines is diagonally
// dominant, hence positive definite.
__global__ void tune_spd_diag_kernel(double* A, const long long* off, const int* n, int count) {
    for (int i = blockIdx.x; i < count; i += gridDim.x) {
        const int ni = n[i];
        for (int d = threadIdx.x; d < ni; d += blockDim.x) A[off[i] + d + (size_t)d * ni] += 2.0 * ni;
    }
}

// Variable-size Cholesky: one persistent launch against one launch per size bucket,
// on 8,192 SPD systems with n on [4, 512] (density ~ n^-1.5) and 1-8 right-hand
// sides, through magma_dposv_vbatched_max_nocheck (both give bit-identical results).
static magma_int_t tune_chol_queue(magma_queue_t q, unsigned seed) {
    const int count = 8192;
    std::vector<int> n(count + 1), r(count + 1);
    std::vector<long long> offA(count), offB(count);
    unsigned long long st = seed * 1000003ull;
    auto unit = [&] {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return double(st >> 11) * (1.0 / 9007199254740992.0);
    };
    const double a = 0.5, b = 1.0 / std::sqrt(512.0);   // 4^-1/2, 512^-1/2: inverse CDF of n^-1.5
    long long na = 0, nb = 0;
    int max_n = 0;
    for (int i = 0; i < count; ++i) {
        const double x = a - unit() * (a - b);
        n[i] = std::min(512, std::max(4, (int)std::lround(1.0 / (x * x))));
        r[i] = 1 + (int)(unit() * 8.0) % 8;
        offA[i] = na;
        offB[i] = nb;
        na += (long long)n[i] * n[i];
        nb += (long long)n[i] * r[i];
        max_n = std::max(max_n, n[i]);
    }
    n[count] = r[count] = 0;
    DevBuf dA, dA0, dB, dP, dI, dO;
    if (!dA.alloc(8 * na) || !dA0.alloc(8 * na) || !dB.alloc(8 * nb) || !dP.alloc(sizeof(double*) * 2 * count) ||
        !dI.alloc(sizeof(int) * 3 * (count + 1)) || !dO.alloc(sizeof(long long) * count))
        return MAGMA_ERR_DEVICE_ALLOC;
    std::vector<double*> ptr(2 * count);
    for (int i = 0; i < count; ++i) {
        ptr[i] = (double*)dA.p + offA[i];
        ptr[count + i] = (double*)dB.p + offB[i];
    }
    int* dn = (int*)dI.p;
    int* dr = dn + count + 1;
    int* dinfo = dr + count + 1;
    cudaMemcpyAsync(dP.p, ptr.data(), sizeof(double*) * 2 * count, cudaMemcpyHostToDevice, q->stream);
    cudaMemcpyAsync(dn, n.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice, q->stream);
    cudaMemcpyAsync(dr, r.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice, q->stream);
    cudaMemcpyAsync(dO.p, offA.data(), sizeof(long long) * count, cudaMemcpyHostToDevice, q->stream);
    tune_fill_kernel<double><<<1024, 256, 0, q->stream>>>((double*)dA0.p, (size_t)na, seed + 1);
    tune_spd_diag_kernel<<<1024, 128, 0, q->stream>>>((double*)dA0.p, (const long long*)dO.p, dn, count);
    tune_fill_kernel<double><<<1024, 256, 0, q->stream>>>((double*)dB.p, (size_t)nb, seed + 2);
    cudaStreamSynchronize(q->stream);
    double** pA = (double**)dP.p;
    double** pB = pA + count;
    float best = 1e30f;
    int best_v = tuning().chol_queue;
    for (int v = 0; v < 2; ++v) {
        tuning_mut().chol_queue = v;
        const float ms = time_ms(q->stream, [&] {
            cudaMemcpyAsync(dA.p, dA0.p, 8 * na, cudaMemcpyDeviceToDevice, q->stream);
            magma_dposv_vbatched_max_nocheck(MagmaLower, dn, dr, pA, dn, pB, dn, dinfo, count, max_n, 8, q);
        }, 3);
        if (cudaGetLastError() != cudaSuccess) return MAGMA_ERR_UNKNOWN;
        if (ms < best) { best = ms; best_v = v; }
    }
    tuning_mut().chol_queue = best_v;
    return MAGMA_SUCCESS;
}

// Variable-size LU: one persistent launch against one launch per size bucket, on 8,192
// diagonally dominant systems with n on [4, 512] (density ~ n^-1.5) and 1-8 right-hand
// sides, through magma_dgesv_vbatched_max_nocheck (both give bit-identical results).
static magma_int_t tune_lu_queue(magma_queue_t q, unsigned seed) {
    const int count = 8192;
    std::vector<int> n(count + 1), r(count + 1);
    std::vector<long long> offA(count), offB(count), offP(count);
    unsigned long long st = seed * 1000003ull;
    auto unit = [&] {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return double(st >> 11) * (1.0 / 9007199254740992.0);
    };
    const double a = 0.5, b = 1.0 / std::sqrt(512.0);
    long long na = 0, nb = 0, np = 0;
    int max_n = 0;
    for (int i = 0; i < count; ++i) {
        const double x = a - unit() * (a - b);
        n[i] = std::min(512, std::max(4, (int)std::lround(1.0 / (x * x))));
        r[i] = 1 + (int)(unit() * 8.0) % 8;
        offA[i] = na;
        offB[i] = nb;
        offP[i] = np;
        na += (long long)n[i] * n[i];
        nb += (long long)n[i] * r[i];
        np += n[i];
        max_n = std::max(max_n, n[i]);
    }
    n[count] = r[count] = 0;
    DevBuf dA, dA0, dB, dP, dI, dO, dV;
    if (!dA.alloc(8 * na) || !dA0.alloc(8 * na) || !dB.alloc(8 * nb) || !dP.alloc(sizeof(void*) * 3 * count) ||
        !dI.alloc(sizeof(int) * 3 * (count + 1)) || !dO.alloc(sizeof(long long) * count) ||
        !dV.alloc(sizeof(int) * np))
        return MAGMA_ERR_DEVICE_ALLOC;
    std::vector<void*> ptr(3 * count);
    for (int i = 0; i < count; ++i) {
        ptr[i] = (double*)dA.p + offA[i];
        ptr[count + i] = (double*)dB.p + offB[i];
        ptr[2 * count + i] = (int*)dV.p + offP[i];
    }
    int* dn = (int*)dI.p;
    int* dr = dn + count + 1;
    int* dinfo = dr + count + 1;
    cudaMemcpyAsync(dP.p, ptr.data(), sizeof(void*) * 3 * count, cudaMemcpyHostToDevice, q->stream);
    cudaMemcpyAsync(dn, n.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice, q->stream);
    cudaMemcpyAsync(dr, r.data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice, q->stream);
    cudaMemcpyAsync(dO.p, offA.data(), sizeof(long long) * count, cudaMemcpyHostToDevice, q->stream);
    tune_fill_kernel<double><<<1024, 256, 0, q->stream>>>((double*)dA0.p, (size_t)na, seed + 1);
    tune_spd_diag_kernel<<<1024, 128, 0, q->stream>>>((double*)dA0.p, (const long long*)dO.p, dn, count);
    tune_fill_kernel<double><<<1024, 256, 0, q->stream>>>((double*)dB.p, (size_t)nb, seed + 2);
    cudaStreamSynchronize(q->stream);
    void** p = (void**)dP.p;
    float best = 1e30f;
    int best_v = tuning().lu_queue;
    for (int v = 0; v < 2; ++v) {
        tuning_mut().lu_queue = v;
        const float ms = time_ms(q->stream, [&] {
            cudaMemcpyAsync(dA.p, dA0.p, 8 * na, cudaMemcpyDeviceToDevice, q->stream);
            magma_dgesv_vbatched_max_nocheck(dn, dr, (double**)p, dn, (int**)(p + 2 * count), (double**)(p + count),
                                             dn, dinfo, count, max_n, 8, q);
        }, 3);
        if (cudaGetLastError() != cudaSuccess) return MAGMA_ERR_UNKNOWN;
        if (ms < best) { best = ms; best_v = v; }
    }
    tuning_mut().lu_queue = best_v;
    return MAGMA_SUCCESS;
}

}  // namespace mb200

using namespace mb200;

extern "C" {

magma_int_t magma_b200_autotune(magma_queue_t queue) {
    if (!queue) return -1;
    cudaSetDevice(queue->device);
    magma_int_t rc = tune_gemm<double>(0, queue, 17);
    if (!rc) rc = tune_gemm<float>(1, queue, 23);
    if (!rc) rc = tune_mixed(queue, 29);
    if (!rc) rc = tune_lu_update(queue, 31);
    if (!rc) rc = tune_chol_queue(queue, 37);
    if (!rc) rc = tune_lu_queue(queue, 41);
    cudaStreamSynchronize(queue->stream);
    return rc;
}

magma_int_t magma_b200_tuning_get(magma_int_t* values, magma_int_t count) {
    if (count < kTuningValues) return kTuningValues;
    to_values(tuning(), values);
    return kTuningValues;
}

magma_int_t magma_b200_tuning_set(const magma_int_t* values, magma_int_t count) {
    TuningTable t = tuning();
    if (!values || !from_values(values, count, t)) return MAGMA_ERR_ILLEGAL_VALUE;
    tuning_mut() = t;
    return MAGMA_SUCCESS;
}

magma_int_t magma_b200_tuning_save(const char* path) {
    if (!path) return MAGMA_ERR_ILLEGAL_VALUE;
    FILE* f = std::fopen(path, "w");
    if (!f) return MAGMA_ERR_UNKNOWN;
    int v[kTuningValues];
    to_values(tuning(), v);
    std::fprintf(f, "magma_b200_tuning_v5\n");
    for (int i = 0; i < kTuningValues; ++i) std::fprintf(f, "%d%c", v[i], i + 1 < kTuningValues ? ' ' : '\n');
    return std::fclose(f) == 0 ? MAGMA_SUCCESS : MAGMA_ERR_UNKNOWN;
}

magma_int_t magma_b200_tuning_load(const char* path) {
    if (!path) return MAGMA_ERR_ILLEGAL_VALUE;
    TuningTable t = tuning();
    if (!load_file(path, t)) return MAGMA_ERR_ILLEGAL_VALUE;
    tuning_mut() = t;
    return MAGMA_SUCCESS;
}

}  // extern "C"
