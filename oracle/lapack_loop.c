/*
 * lapack_loop.c -- TEST AND BASELINE INFRASTRUCTURE ONLY. The reference's own
 * CPU implementation of the batched path: an OpenMP loop over instances that
 * calls host LAPACK once per instance with one BLAS thread per OpenMP thread,
 * exactly as MAGMA's testers time it (testing/testing_zgetrf_batched.cpp:188-206:
 * "#pragma omp parallel for schedule(dynamic)" + magma_set_lapack_numthreads(1)).
 *
 * The LAPACK is the one in this image, OpenBLAS 0.3.30 from scipy 1.18.1
 * (libscipy_openblas, LP64, symbols prefixed "scipy_"); its path is handed to
 * lapack_loop_init() at run time and the library is dlopen'ed. Used by the
 * tests to pin the oracle restatement and by bench.py as the CPU baseline
 * (the reference arm). Never linked into libmagma_b200.
 */
#include <dlfcn.h>
#include <stddef.h>
#include <omp.h>

typedef void (*getrf_t)(const int*, const int*, double*, const int*, int*, int*);
typedef void (*getrs_t)(const char*, const int*, const int*, const double*, const int*, const int*,
                        double*, const int*, int*, size_t);
typedef void (*gesv_t)(const int*, const int*, double*, const int*, int*, double*, const int*, int*);
typedef void (*potrf_t)(const char*, const int*, double*, const int*, int*, size_t);
typedef void (*potrs_t)(const char*, const int*, const int*, const double*, const int*, double*,
                        const int*, int*, size_t);
typedef void (*dgemm_t)(const char*, const char*, const int*, const int*, const int*, const double*,
                        const double*, const int*, const double*, const int*, const double*, double*,
                        const int*, size_t, size_t);
typedef void (*sgemm_t)(const char*, const char*, const int*, const int*, const int*, const float*,
                        const float*, const int*, const float*, const int*, const float*, float*,
                        const int*, size_t, size_t);
typedef void (*dsgesv_t)(const int*, const int*, double*, const int*, int*, const double*, const int*,
                         double*, const int*, double*, float*, int*, int*);
typedef void (*geqrf_t)(const int*, const int*, double*, const int*, double*, double*, const int*, int*);
typedef void (*getri_t)(const int*, double*, const int*, const int*, double*, const int*, int*);
typedef void (*trxm_t)(const char*, const char*, const char*, const char*, const int*, const int*, const double*,
                       const double*, const int*, double*, const int*, size_t, size_t, size_t, size_t);
typedef void (*syrk_t)(const char*, const char*, const int*, const int*, const double*, const double*, const int*,
                       const double*, double*, const int*, size_t, size_t);
typedef void (*setthreads_t)(int);

static getrf_t p_dgetrf;
static getrs_t p_dgetrs;
static gesv_t p_dgesv;
static potrf_t p_dpotrf;
static potrs_t p_dpotrs;
static dgemm_t p_dgemm;
static sgemm_t p_sgemm;
static dsgesv_t p_dsgesv;
static geqrf_t p_dgeqrf;
static getri_t p_dgetri;
static trxm_t p_dtrsm, p_dtrmm;
static syrk_t p_dsyrk;
static setthreads_t p_setthreads;

/* Returns 0 on success, -1 if the library or a symbol is missing. */
int lapack_loop_init(const char* path) {
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return -1;
    p_dgetrf = (getrf_t)dlsym(h, "scipy_dgetrf_");
    p_dgetrs = (getrs_t)dlsym(h, "scipy_dgetrs_");
    p_dgesv = (gesv_t)dlsym(h, "scipy_dgesv_");
    p_dpotrf = (potrf_t)dlsym(h, "scipy_dpotrf_");
    p_dpotrs = (potrs_t)dlsym(h, "scipy_dpotrs_");
    p_dgemm = (dgemm_t)dlsym(h, "scipy_dgemm_");
    p_sgemm = (sgemm_t)dlsym(h, "scipy_sgemm_");
    p_dsgesv = (dsgesv_t)dlsym(h, "scipy_dsgesv_");
    p_dgeqrf = (geqrf_t)dlsym(h, "scipy_dgeqrf_");
    p_dgetri = (getri_t)dlsym(h, "scipy_dgetri_");
    p_dtrsm = (trxm_t)dlsym(h, "scipy_dtrsm_");
    p_dtrmm = (trxm_t)dlsym(h, "scipy_dtrmm_");
    p_dsyrk = (syrk_t)dlsym(h, "scipy_dsyrk_");
    p_setthreads = (setthreads_t)dlsym(h, "scipy_openblas_set_num_threads");
    if (!p_dgetrf || !p_dgetrs || !p_dgesv || !p_dpotrf || !p_dpotrs || !p_dgemm || !p_sgemm ||
        !p_dsgesv || !p_dgeqrf || !p_dgetri || !p_dtrsm || !p_dtrmm || !p_dsyrk ||
        !p_setthreads)
        return -1;
    p_setthreads(1);
    return 0;
}

int lapack_loop_max_threads(void) { return omp_get_max_threads(); }

/* dgetrf per instance (testing_zgetrf_batched.cpp:200). */
void ref_dgetrf_batched(int m, int n, double* A, int lda, long sA, int* ipiv, long sP, int* info,
                        int batch, int nthreads) {
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i)
        p_dgetrf(&m, &n, A + (size_t)i * sA, &lda, ipiv + (size_t)i * sP, info + i);
}

void ref_dgetrs_batched(int trans, int n, int nrhs, const double* A, int lda, long sA, const int* ipiv,
                        long sP, double* B, int ldb, long sB, int batch, int nthreads) {
    const char t = trans ? 'T' : 'N';
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i) {
        int info = 0;
        p_dgetrs(&t, &n, &nrhs, A + (size_t)i * sA, &lda, ipiv + (size_t)i * sP, B + (size_t)i * sB,
                 &ldb, &info, 1);
    }
}

/* dgesv per instance (testing_zgesv_batched.cpp:171). */
void ref_dgesv_batched(int n, int nrhs, double* A, int lda, long sA, int* ipiv, long sP, double* B,
                       int ldb, long sB, int* info, int batch, int nthreads) {
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i)
        p_dgesv(&n, &nrhs, A + (size_t)i * sA, &lda, ipiv + (size_t)i * sP, B + (size_t)i * sB, &ldb,
                info + i);
}

/* Variable-size dpotrf (+ dpotrs) per instance (testing_zpotrf_vbatched.cpp:166). */
void ref_dposv_vbatched(const int* n, const int* nrhs, double* const* A, const int* lda,
                        double* const* B, const int* ldb, int* info, int batch, int do_solve,
                        int nthreads) {
    const char lo = 'L';
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i) {
        p_dpotrf(&lo, &n[i], A[i], &lda[i], &info[i], 1);
        if (do_solve && info[i] == 0) {
            int inf2 = 0;
            p_dpotrs(&lo, &n[i], &nrhs[i], A[i], &lda[i], B[i], &ldb[i], &inf2, 1);
        }
    }
}

/* Variable-size gemm per instance (testing_zgemm_vbatched.cpp:293). */
void ref_dgemm_vbatched(int ta, int tb, const int* m, const int* n, const int* k, double alpha,
                        double* const* A, const int* lda, double* const* B, const int* ldb, double beta,
                        double* const* C, const int* ldc, int batch, int nthreads) {
    const char a = ta ? 'T' : 'N', b = tb ? 'T' : 'N';
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i)
        p_dgemm(&a, &b, &m[i], &n[i], &k[i], &alpha, A[i], &lda[i], B[i], &ldb[i], &beta, C[i], &ldc[i], 1, 1);
}

void ref_sgemm_vbatched(int ta, int tb, const int* m, const int* n, const int* k, float alpha,
                        float* const* A, const int* lda, float* const* B, const int* ldb, float beta,
                        float* const* C, const int* ldc, int batch, int nthreads) {
    const char a = ta ? 'T' : 'N', b = tb ? 'T' : 'N';
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i)
        p_sgemm(&a, &b, &m[i], &n[i], &k[i], &alpha, A[i], &lda[i], B[i], &ldb[i], &beta, C[i], &ldc[i], 1, 1);
}

/* LAPACK's own mixed-precision solver per instance (the CPU counterpart of
 * magma_dsgesv_gpu, src/zcgesv_gpu.cpp:144). iter follows LAPACK dsgesv. */
void ref_dsgesv_batched(int n, int nrhs, double* A, int lda, long sA, int* ipiv, long sP, const double* B,
                        int ldb, long sB, double* X, int ldx, long sX, int* iter, int* info, int batch,
                        int nthreads) {
#pragma omp parallel num_threads(nthreads)
    {
        double* work = (double*)__builtin_alloca(sizeof(double) * (size_t)n * nrhs);
        float* swork = (float*)__builtin_alloca(sizeof(float) * (size_t)n * (n + nrhs));
#pragma omp for schedule(dynamic)
        for (int i = 0; i < batch; ++i)
            p_dsgesv(&n, &nrhs, A + (size_t)i * sA, &lda, ipiv + (size_t)i * sP, B + (size_t)i * sB, &ldb,
                     X + (size_t)i * sX, &ldx, work, swork, iter + i, info + i);
    }
}

/* dgeqrf per instance (testing_zgeqrf_batched.cpp:218-230). */
void ref_dgeqrf_batched(int m, int n, double* A, int lda, long sA, double* tau, long sT, int batch,
                        int nthreads) {
#pragma omp parallel num_threads(nthreads)
    {
        int lwork = 64 * (n > 0 ? n : 1);
        double* work = (double*)__builtin_alloca(sizeof(double) * (size_t)lwork);
#pragma omp for schedule(dynamic)
        for (int i = 0; i < batch; ++i) {
            int info = 0;
            p_dgeqrf(&m, &n, A + (size_t)i * sA, &lda, tau + (size_t)i * sT, work, &lwork, &info);
        }
    }
}

/* dgetrf + dgetri per instance, in place (testing_zgetri_batched.cpp:140-160). */
void ref_dgetri_batched(int n, double* A, int lda, long sA, int* ipiv, long sP, int* info, int batch,
                        int nthreads) {
#pragma omp parallel num_threads(nthreads)
    {
        int lwork = 64 * (n > 0 ? n : 1);
        double* work = (double*)__builtin_alloca(sizeof(double) * (size_t)lwork);
#pragma omp for schedule(dynamic)
        for (int i = 0; i < batch; ++i) {
            p_dgetrf(&n, &n, A + (size_t)i * sA, &lda, ipiv + (size_t)i * sP, info + i);
            int inf2 = 0;
            if (info[i] == 0) p_dgetri(&n, A + (size_t)i * sA, &lda, ipiv + (size_t)i * sP, work, &lwork, &inf2);
        }
    }
}

/* dtrsm (solve != 0) or dtrmm per instance (testing_ztrsm_vbatched.cpp:327, testing_ztrmm_vbatched.cpp:238). */
void ref_dtri_vbatched(int solve, int left, int lower, int trans, int unit, const int* m, const int* n, double alpha,
                       double* const* A, const int* lda, double* const* B, const int* ldb, int batch, int nthreads) {
    const char sd = left ? 'L' : 'R', ul = lower ? 'L' : 'U', tr = trans ? 'T' : 'N', dg = unit ? 'U' : 'N';
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i) {
        if (m[i] <= 0 || n[i] <= 0) continue;
        if (solve) p_dtrsm(&sd, &ul, &tr, &dg, &m[i], &n[i], &alpha, A[i], &lda[i], B[i], &ldb[i], 1, 1, 1, 1);
        else p_dtrmm(&sd, &ul, &tr, &dg, &m[i], &n[i], &alpha, A[i], &lda[i], B[i], &ldb[i], 1, 1, 1, 1);
    }
}

/* dsyrk per instance (testing_zsyrk_vbatched.cpp:244). */
void ref_dsyrk_vbatched(int lower, int trans, const int* n, const int* k, double alpha, double* const* A,
                        const int* lda, double beta, double* const* C, const int* ldc, int batch, int nthreads) {
    const char ul = lower ? 'L' : 'U', tr = trans ? 'T' : 'N';
#pragma omp parallel for schedule(dynamic) num_threads(nthreads)
    for (int i = 0; i < batch; ++i) {
        if (n[i] <= 0) continue;
        p_dsyrk(&ul, &tr, &n[i], &k[i], &alpha, A[i], &lda[i], &beta, C[i], &ldc[i], 1, 1);
    }
}
