/*
 * lapack_oracle.c -- TEST INFRASTRUCTURE ONLY. CPU restatement of the LAPACK
 * algorithms that MAGMA's batched testers use as their correctness oracle.
 * Nothing in the shipped library links or calls this file; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
 *
 * The reference's CPU oracle is host LAPACK, called per instance from the
 * testers (testing/testing_zgetrf_batched.cpp:188-206 dgetrf,
 * testing/testing_zgesv_batched.cpp:171 dgesv,
 * testing/testing_zpotrf_vbatched.cpp:166 dpotrf,
 * testing/testing_zgemm_vbatched.cpp:293 dgemm). LAPACK is a third-party
 * dependency absent from the reference tree; in this image it is OpenBLAS
 * 0.3.30 bundled with scipy 1.18.1 (libscipy_openblas, LP64). This file
 * restates the published netlib algorithms (LAPACK 3.x dgetf2 / dgetrs /
 * dpotf2 / dpotrs, reference BLAS dger / dtrsm / dgemm) with every
 * multiply-add written as an explicit fma(), so that a GPU kernel doing the
 * same operations in the same order can be compared bit for bit. It is
 * pinned against the real OpenBLAS on committed golden vectors
 * (tests/golden/, made by tests/golden/make_golden.py).
 *
 * Deliberate, documented departures from netlib:
 *  - reference BLAS skips updates whose multiplier is exactly zero
 *    (DGER "IF (Y(JY).NE.ZERO)", DTRSM "IF (B(K,J).NE.ZERO)"); the skip only
 *    changes the sign of zero results or NaN propagation, so it is omitted;
 *  - IDAMAX with NaNs: a NaN magnitude ranks below every number (netlib
 *    returns a leading NaN). Finite inputs are unaffected.
 *
 * Compile: make -C oracle   (gcc -O2 -fopenmp -ffp-contract=off)
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <stddef.h>
#include <string.h>

#define A_(i, j) a[(size_t)(i) + (size_t)(j) * (size_t)lda]
#define B_(i, j) b[(size_t)(i) + (size_t)(j) * (size_t)ldb]

static double pivot_key(double x) {
    double v = fabs(x);
    return (v != v) ? -0.5 : v;
}

/* LAPACK 3.x dgetf2: unblocked right-looking LU with partial pivoting
 * (pivot = 0: no search, the diagonal is the pivot).
 * ipiv is 1-based; info = first zero pivot (1-based) or 0. */
static void getf2(int m, int n, double* a, int lda, int* ipiv, int* info, int pivot) {
    *info = 0;
    const int kmax = m < n ? m : n;
    for (int j = 0; j < kmax; ++j) {
        int jp = j;
        double best = pivot_key(A_(j, j));
        for (int i = j + 1; pivot && i < m; ++i) {
            double v = pivot_key(A_(i, j));
            if (v > best) { best = v; jp = i; }
        }
        ipiv[j] = jp + 1;
        const double piv = A_(jp, j);
        if (piv != 0.0) {
            if (jp != j) {
                for (int c = 0; c < n; ++c) { double t = A_(j, c); A_(j, c) = A_(jp, c); A_(jp, c) = t; }
            }
            if (fabs(piv) >= DBL_MIN) {
                const double r = 1.0 / piv;
                for (int i = j + 1; i < m; ++i) A_(i, j) = A_(i, j) * r;
            } else {
                for (int i = j + 1; i < m; ++i) A_(i, j) = A_(i, j) / piv;
            }
        } else if (*info == 0) {
            *info = j + 1;
        }
        if (j < kmax - 1) {
            for (int c = j + 1; c < n; ++c) {
                const double u = A_(j, c);
                for (int i = j + 1; i < m; ++i) A_(i, c) = fma(A_(i, j), -u, A_(i, c));
            }
        }
    }
}

void oracle_dgetf2(int m, int n, double* a, int lda, int* ipiv, int* info) { getf2(m, n, a, lda, ipiv, info, 1); }

/* The same elimination without pivoting (MAGMA's getrf_nopiv): step j's pivot is
 * the diagonal entry; ipiv is filled with the identity sequence. */
void oracle_dgetf2_nopiv(int m, int n, double* a, int lda, int* ipiv, int* info) {
    getf2(m, n, a, lda, ipiv, info, 0);
}

void oracle_dgetrf_nopiv_batched(int m, int n, double* A, int lda, long strideA, int* ipiv, long strideP,
                                 int* info, int batch) {
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < batch; ++i)
        oracle_dgetf2_nopiv(m, n, A + (size_t)i * strideA, lda, ipiv + (size_t)i * strideP, info + i);
}

/* The reference's QR tester checks magma_zgeqrf_batched against host LAPACK zgeqrf, one
 * instance at a time (testing/testing_zgeqrf_batched.cpp:224).
 * LAPACK 3.x dgeqr2 (Householder QR: dlarfg, then dlarf on the trailing columns), with
 * the summation order of the batched path written out: the rows of a column are dealt
 * to P lanes (row r to lane r mod P, P = 1, 2, 4, 8, 16 for m <= 16, 32, 64, 512, 1024); each
 * lane sums its rows in ascending order with fma, and the P partial sums are added as
 * a pairwise tree ((x0+x1)+(x2+x3))+... . For column k:
 *   xs = ||A(k+1:m, k)||^2 in that order, beta = -sign(alpha) sqrt(fma(alpha, alpha, xs)),
 *   tau = (beta - alpha) / beta, v_r = A(r,k) * (1 / (alpha - beta)); tau = 0 when xs = 0;
 *   with s_r = 0 (r < k), 1 (r = k), v_r (r > k) and t_r = -tau * s_r, every trailing
 *   column j takes w = sum_r s_r A(r,j) (all m rows, in that order) and
 *   A(r,j) = fma(t_r, w, A(r,j)) for all m rows (rows above k change by an exact zero).
 * Against LAPACK this differs by rounding only (and the sign of exact zeros); dnrm2's
 * scaling and dlapy2's guard are omitted (entries far inside [1e-150, 1e150]). */
static int qr_lanes(int m) { return m <= 16 ? 1 : m <= 32 ? 2 : m <= 64 ? 4 : m <= 512 ? 8 : 16; }

static double tree_sum(double* x, int P) {
    for (int h = 1; h < P; h *= 2)
        for (int p = 0; p < P; p += 2 * h) x[p] = x[p] + x[p + h];
    return x[0];
}

void oracle_dgeqr2(int m, int n, double* a, int lda, double* tau) {
    const int kmax = m < n ? m : n, P = qr_lanes(m);
    double part[32];
    double* sv = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double* st = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    for (int k = 0; k < kmax; ++k) {
        for (int p = 0; p < P; ++p) part[p] = 0.0;
        for (int r = k + 1; r < m; ++r) part[r % P] = fma(A_(r, k), A_(r, k), part[r % P]);
        const double xs = tree_sum(part, P);
        const double alpha = A_(k, k);
        double t = 0.0, beta = alpha, scal = 1.0;
        if (xs > 0.0) {
            beta = -copysign(sqrt(fma(alpha, alpha, xs)), alpha);
            t = (beta - alpha) / beta;
            scal = 1.0 / (alpha - beta);
        }
        for (int r = 0; r < m; ++r) sv[r] = r < k ? 0.0 : r == k ? 1.0 : A_(r, k) * scal;
        for (int r = 0; r < m; ++r) st[r] = -t * sv[r];
        tau[k] = t;
        if (t == 0.0) continue;
        for (int r = k + 1; r < m; ++r) A_(r, k) = sv[r];
        A_(k, k) = beta;
        for (int j = k + 1; j < n; ++j) {
            for (int p = 0; p < P; ++p) part[p] = 0.0;
            for (int r = 0; r < m; ++r) part[r % P] = fma(sv[r], A_(r, j), part[r % P]);
            const double w = tree_sum(part, P);
            for (int r = 0; r < m; ++r) A_(r, j) = fma(st[r], w, A_(r, j));
        }
    }
    free(sv);
    free(st);
}

void oracle_dgeqrf_batched(int m, int n, double* A, int lda, long strideA, double* tau, long strideT, int batch) {
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < batch; ++i)
        oracle_dgeqr2(m, n, A + (size_t)i * strideA, lda, tau + (size_t)i * strideT);
}

/* LAPACK dlaswp on the rows of B: forward (k ascending) or inverse. */
static void laswp(int n, int nrhs, double* b, int ldb, const int* ipiv, int inverse) {
    for (int t = 0; t < n; ++t) {
        const int k = inverse ? n - 1 - t : t;
        const int p = ipiv[k] - 1;
        if (p != k)
            for (int c = 0; c < nrhs; ++c) { double x = B_(k, c); B_(k, c) = B_(p, c); B_(p, c) = x; }
    }
}

/* LAPACK dgetrs with reference-BLAS dtrsm loop orders.
 * trans = 0: A X = B;  trans != 0: A^T X = B. */
void oracle_dgetrs(int trans, int n, int nrhs, const double* a, int lda, const int* ipiv,
                   double* b, int ldb) {
    if (!trans) {
        laswp(n, nrhs, b, ldb, ipiv, 0);
        for (int c = 0; c < nrhs; ++c) {
            /* DTRSM Left Lower NoTrans Unit */
            for (int k = 0; k < n; ++k)
                for (int i = k + 1; i < n; ++i) B_(i, c) = fma(-B_(k, c), A_(i, k), B_(i, c));
            /* DTRSM Left Upper NoTrans NonUnit */
            for (int k = n - 1; k >= 0; --k) {
                B_(k, c) = B_(k, c) / A_(k, k);
                for (int i = 0; i < k; ++i) B_(i, c) = fma(-B_(k, c), A_(i, k), B_(i, c));
            }
        }
    } else {
        for (int c = 0; c < nrhs; ++c) {
            /* DTRSM Left Upper Trans NonUnit: dot-product form, k ascending */
            for (int i = 0; i < n; ++i) {
                double t = B_(i, c);
                for (int k = 0; k < i; ++k) t = fma(-A_(k, i), B_(k, c), t);
                B_(i, c) = t / A_(i, i);
            }
            /* DTRSM Left Lower Trans Unit: i descending, k ascending */
            for (int i = n - 1; i >= 0; --i) {
                double t = B_(i, c);
                for (int k = i + 1; k < n; ++k) t = fma(-A_(k, i), B_(k, c), t);
                B_(i, c) = t;
            }
        }
        laswp(n, nrhs, b, ldb, ipiv, 1);
    }
}

/* ---------------------------------------------------------------------------
 * Batched drivers over contiguous batches (instance i at base + i*stride),
 * one instance per OpenMP iteration as in testing_zgetrf_batched.cpp:188-206. */
void oracle_dgetrf_batched(int m, int n, double* A, int lda, long strideA, int* ipiv, long strideP,
                           int* info, int batch) {
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < batch; ++i)
        oracle_dgetf2(m, n, A + (size_t)i * strideA, lda, ipiv + (size_t)i * strideP, info + i);
}

void oracle_dgetrs_batched(int trans, int n, int nrhs, const double* A, int lda, long strideA,
                           const int* ipiv, long strideP, double* B, int ldb, long strideB, int batch) {
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < batch; ++i)
        oracle_dgetrs(trans, n, nrhs, A + (size_t)i * strideA, lda, ipiv + (size_t)i * strideP,
                      B + (size_t)i * strideB, ldb);
}

/* MAGMA's batched gesv solves every instance whatever its info
 * (src/zgesv_batched.cpp:127-145). */
void oracle_dgesv_batched(int n, int nrhs, double* A, int lda, long strideA, int* ipiv, long strideP,
                          double* B, int ldb, long strideB, int* info, int batch) {
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < batch; ++i) {
        double* Ai = A + (size_t)i * strideA;
        int* pi = ipiv + (size_t)i * strideP;
        oracle_dgetf2(n, n, Ai, lda, pi, info + i);
        oracle_dgetrs(0, n, nrhs, Ai, lda, pi, B + (size_t)i * strideB, ldb);
    }
}

/* ---------------------------------------------------------------------------
 * Cholesky. LAPACK dpotrf / dpotf2 (uplo = 'L'): A = L L^T. The reference's
 * GPU path supports Lower only (src/zpotf2_vbatched.cpp:32-34). This
 * restatement uses the outer-product (right-looking) form of the same
 * factorisation: for k = 0..n-1
 *     d = A(k,k); if !(d > 0) -> info = k+1, A(k,k) keeps d, stop  (dpotf2:
 *         "IF( AJJ.LE.ZERO.OR.DISNAN( AJJ ) )", A(J,J) = AJJ, INFO = J)
 *     A(k,k) = sqrt(d); A(k+1:n,k) *= 1/A(k,k)           (dpotf2: DSCAL by ONE/AJJ)
 *     A(i,j) = fma(-A(i,k), A(j,k), A(i,j)) for k < j <= i (rank-1 update)
 * It differs from dpotf2's dot-product form only in the summation order, and
 * is pinned to OpenBLAS's dpotrf on the golden vectors within tolerance.
 * Upper: the same on the transpose (A = U^T U with U = L^T).
 */
void oracle_dpotrf(int upper, int n, double* a, int lda, int* info) {
    *info = 0;
#define AL(i, j) (*(upper ? &A_(j, i) : &A_(i, j)))
    for (int k = 0; k < n; ++k) {
        double d = AL(k, k);
        if (!(d > 0.0)) { *info = k + 1; return; }
        d = sqrt(d);
        AL(k, k) = d;
        const double r = 1.0 / d;
        for (int i = k + 1; i < n; ++i) AL(i, k) = AL(i, k) * r;
        for (int j = k + 1; j < n; ++j)
            for (int i = j; i < n; ++i) AL(i, j) = fma(-AL(i, k), AL(j, k), AL(i, j));
    }
#undef AL
}

/* LAPACK dpotrs: L y = b (column sweep, reference DTRSM Left Lower NoTrans
 * NonUnit), then L^T x = y by the column sweep of the upper-triangular solve
 * with U = L^T (reference DTRSM Left Upper NoTrans NonUnit loop order), except
 * that b(k) is multiplied by the correctly rounded 1/L(k,k) where DTRSM divides
 * (the batched kernels' form: no division on the sweep's dependency chain). */
void oracle_dpotrs(int upper, int n, int nrhs, const double* a, int lda, double* b, int ldb) {
#define LL(i, j) (*(upper ? &A_(j, i) : &A_(i, j)))
    for (int c = 0; c < nrhs; ++c) {
        for (int k = 0; k < n; ++k) {
            B_(k, c) = B_(k, c) * (1.0 / LL(k, k));
            for (int i = k + 1; i < n; ++i) B_(i, c) = fma(-B_(k, c), LL(i, k), B_(i, c));
        }
        for (int k = n - 1; k >= 0; --k) {
            B_(k, c) = B_(k, c) * (1.0 / LL(k, k));
            for (int i = 0; i < k; ++i) B_(i, c) = fma(-B_(k, c), LL(k, i), B_(i, c));
        }
    }
#undef LL
}

/* Variable-size batched Cholesky over pointer lists (one instance per iteration). */
void oracle_dposv_vbatched(int upper, const int* n, const int* nrhs, double* const* A, const int* lda,
                           double* const* B, const int* ldb, int* info, int batch, int do_solve) {
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < batch; ++i) {
        oracle_dpotrf(upper, n[i], A[i], lda[i], &info[i]);
        if (do_solve) oracle_dpotrs(upper, n[i], nrhs[i], A[i], lda[i], B[i], ldb[i]);
    }
}

/* The reference's testers check the batched triangular routines against host BLAS:
 * ztrsm (testing/testing_ztrsm_vbatched.cpp:327) and ztrmm
 * (testing/testing_ztrmm_vbatched.cpp:238), one instance at a time.
 * Triangular solve / multiply (BLAS dtrsm / dtrmm semantics) in the batched kernels'
 * order of operations. The call is seen as a left problem on T (nr x nr) and X
 * (nr x nc): side Left: T = op(A), X = B; side Right: T = op(A)^T, X = B^T. Rows are
 * renumbered q (q = i, or nr-1-i) so that T is lower in q for the solve and upper for
 * the multiply. Per element:
 *   solve:    s = alpha*b; s = fma(-T(q,q'), x(q'), s) for q' < q ascending; x = s * (1/T(q,q))
 *             (unit diagonal: the reciprocal is 1);
 *   multiply: s = 0; s = fma(T(q,q'), b(q'), s) for q' >= q ascending; x = alpha * s.
 * BLAS itself divides by the diagonal and sums in its own order: the two agree to
 * rounding. alpha = 0 sets X to zero. */
void oracle_dtri(int solve, int left, int lowerA, int transA, int unit, int m, int n, double alpha,
                 const double* A, int lda, double* B, int ldb) {
    const int nr = left ? m : n, nc = left ? n : m;
    const int op_lower = (lowerA != 0) != (transA != 0);
    const int t_lower = left ? op_lower : !op_lower;
    const int tt = left ? (transA != 0) : !(transA != 0);
    const int bt = !left;
    const int flip = solve ? !t_lower : t_lower;
#define TRI_ROW(q) (flip ? nr - 1 - (q) : (q))
#define TRI_T(q, qk) (tt ? A[TRI_ROW(qk) + (size_t)TRI_ROW(q) * lda] : A[TRI_ROW(q) + (size_t)TRI_ROW(qk) * lda])
#define TRI_X(q, c) (*(bt ? &B[(c) + (size_t)TRI_ROW(q) * ldb] : &B[TRI_ROW(q) + (size_t)(c) * ldb]))
    if (alpha == 0.0) {
        for (int c = 0; c < nc; ++c)
            for (int q = 0; q < nr; ++q) TRI_X(q, c) = 0.0;
        return;
    }
    for (int c = 0; c < nc; ++c) {
        for (int q = 0; q < nr; ++q) {
            double s;
            if (solve) {
                s = alpha * TRI_X(q, c);
                for (int qk = 0; qk < q; ++qk) s = fma(-TRI_T(q, qk), TRI_X(qk, c), s);
                const double rcp = unit ? 1.0 : 1.0 / TRI_T(q, q);
                TRI_X(q, c) = s * rcp;
            } else {
                s = 0.0;
                for (int qk = q; qk < nr; ++qk) {
                    const double t = (qk == q && unit) ? 1.0 : TRI_T(q, qk);
                    s = fma(t, TRI_X(qk, c), s);
                }
                TRI_X(q, c) = alpha * s;
            }
        }
    }
#undef TRI_ROW
#undef TRI_T
#undef TRI_X
}
