/* A C caller of the host-memory pipeline (include/magma_b200.h): systems generated in
 * page-locked host memory, solved by magma_b200_host_solve in chunks, checked on the
 * host. Built and run by tests/test_host_c_gpu.py; prints one line:
 *   ok <kind> <batch> <n> <max backward error> <sum of iter or pivot checks>
 * and exits 0, or prints the failure and exits 1. Diagonally dominant systems: the
 * mixed solve refines (iter >= 0) and the FP64 solve keeps the diagonal pivots. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "magma_b200.h"

static double uni(unsigned long long* s) {   /* splitmix64 -> [-1, 1) */
    unsigned long long z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

int main(int argc, char** argv) {
    const int kind = argc > 1 ? atoi(argv[1]) : MAGMA_B200_HOST_DSGESV;
    const magma_int_t batch = argc > 2 ? atoi(argv[2]) : 300, n = argc > 3 ? atoi(argv[3]) : 96, nrhs = 3;
    const magma_int_t chunks = 5;
    if (magma_init() != MAGMA_SUCCESS) { printf("magma_init failed\n"); return 1; }
    magma_queue_t q;
    magma_queue_create(0, &q);
    const size_t sa = (size_t)n * n, sb = (size_t)n * nrhs;
    double *hA, *hB, *hX;
    magma_int_t *hI, *hInfo;
    const size_t ni = kind == MAGMA_B200_HOST_DSGESV ? (size_t)batch : (size_t)batch * n;
    if (magma_malloc_pinned((void**)&hA, 8 * sa * batch) || magma_malloc_pinned((void**)&hB, 8 * sb * batch) ||
        magma_malloc_pinned((void**)&hX, 8 * sb * batch) || magma_malloc_pinned((void**)&hI, sizeof(magma_int_t) * ni) ||
        magma_malloc_pinned((void**)&hInfo, sizeof(magma_int_t) * batch)) {
        printf("magma_malloc_pinned failed\n");
        return 1;
    }
    unsigned long long seed = 12345;
    for (size_t i = 0; i < sa * batch; ++i) hA[i] = uni(&seed);
    for (magma_int_t b = 0; b < batch; ++b)
        for (magma_int_t d = 0; d < n; ++d) hA[b * sa + d + (size_t)d * n] += n;   /* diagonally dominant */
    for (size_t i = 0; i < sb * batch; ++i) hB[i] = uni(&seed);
    magma_b200_host_solver_t s;
    magma_int_t rc = magma_b200_host_solver_create(kind, batch, n, nrhs, n, n, chunks, q, &s);
    if (rc != MAGMA_SUCCESS) { printf("create failed: %d\n", (int)rc); return 1; }
    for (int rep = 0; rep < 2; ++rep) {   /* the staging buffers are reused */
        for (size_t i = 0; i < sb * batch; ++i) hX[i] = NAN;
        rc = magma_b200_host_solve(s, hA, hB, hX, hI, hInfo);
        magma_queue_sync(q);
        if (rc != MAGMA_SUCCESS) { printf("solve failed: %d\n", (int)rc); return 1; }
    }
    double worst = 0.0;
    long checks = 0;
    for (magma_int_t b = 0; b < batch; ++b) {
        const double *A = hA + b * sa, *B = hB + b * sb, *X = hX + b * sb;
        if (hInfo[b] != 0) { printf("info[%d] = %d\n", (int)b, (int)hInfo[b]); return 1; }
        double anorm = 0.0;
        for (magma_int_t i = 0; i < n; ++i) {
            double r = 0.0;
            for (magma_int_t j = 0; j < n; ++j) r += fabs(A[i + j * n]);
            if (r > anorm) anorm = r;
        }
        for (magma_int_t c = 0; c < nrhs; ++c) {
            double rn = 0.0, xn = 0.0, bn = 0.0;
            for (magma_int_t i = 0; i < n; ++i) {
                double r = B[i + c * n];
                for (magma_int_t j = 0; j < n; ++j) r -= A[i + j * n] * X[j + c * n];
                if (fabs(r) > rn) rn = fabs(r);
                if (fabs(X[i + c * n]) > xn) xn = fabs(X[i + c * n]);
                if (fabs(B[i + c * n]) > bn) bn = fabs(B[i + c * n]);
            }
            const double be = rn / (anorm * xn + bn);
            if (!(be <= worst)) worst = be;   /* NaN propagates */
        }
        if (kind == MAGMA_B200_HOST_DSGESV) {
            if (hI[b] < 0) { printf("iter[%d] = %d\n", (int)b, (int)hI[b]); return 1; }
            checks += hI[b];
        } else {
            for (magma_int_t k = 0; k < n; ++k) checks += hI[b * n + k] == k + 1;   /* diagonal pivots */
        }
    }
    magma_b200_host_solver_destroy(s);
    magma_free_pinned(hA); magma_free_pinned(hB); magma_free_pinned(hX); magma_free_pinned(hI); magma_free_pinned(hInfo);
    magma_queue_destroy(q);
    magma_finalize();
    if (!(worst <= 1e-14)) { printf("backward error %g\n", worst); return 1; }
    printf("ok %d %d %d %.3g %ld\n", kind, (int)batch, (int)n, worst, checks);
    return 0;
}
