/*
 * magma_b200.h -- public C interface of libmagma_b200.
 *
 * libmagma_b200 is a B200 (sm_100a) implementation of MAGMA's batched
 * small-matrix dense path. Each entry point below keeps the name, argument
 * order, argument meaning and error behaviour of the MAGMA 2.2 routine it
 * replaces (cited per declaration as reference file:line), so a caller that
 * was built against MAGMA relinks against this library unchanged.
 *
 * Conventions shared by every batched routine (as in MAGMA):
 *   - all arrays (pointer arrays, size arrays, ipiv, info, matrices) are
 *     DEVICE memory owned by the caller; matrices are column-major;
 *   - ipiv entries are 1-based row indices in LAPACK's swap-sequence form;
 *   - a negative return value -i means argument i was illegal (reported
 *     through magma_xerbla); numerical failures are reported per instance in
 *     info_array (>0: 1-based index of the first zero pivot / non-positive
 *     leading minor);
 *   - work is enqueued on the queue's CUDA stream. Unlike the reference these
 *     routines do not synchronize before returning (no cudaMalloc, no host
 *     round trip on the call path), so results are visible after
 *     magma_queue_sync(queue), exactly as after the reference's own return.
 *   - vbatched size arrays have batchCount+1 entries; the last one is scratch
 *     (magmablas/zgemm_vbatched.cpp:146-149).
 */
#ifndef MAGMA_B200_H
#define MAGMA_B200_H

#include "magma_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Runtime (reference: interface_cuda/interface.cpp, interface_cuda/alloc.cpp,
 * interface_cuda/copy_v2.cpp, control/xerbla.cpp)
 * ---------------------------------------------------------------------- */

/* interface_cuda/interface.cpp:168 */
magma_int_t magma_init(void);
/* interface_cuda/interface.cpp:246 */
magma_int_t magma_finalize(void);
/* interface_cuda/error.cpp:112 */
const char* magma_strerror(magma_int_t error);
/* control/xerbla.cpp:51 */
void magma_xerbla(const char* srname, magma_int_t neg_info);

/* interface_cuda/interface.cpp:546 (magma_getdevice), :567 (magma_setdevice) */
void magma_getdevice(magma_device_t* dev);
void magma_setdevice(magma_device_t dev);

/* interface_cuda/alloc.cpp:60 (magma_malloc), :93 (magma_free_internal) */
magma_int_t magma_malloc(magma_ptr* ptr_ptr, size_t bytes);
magma_int_t magma_free_internal(magma_ptr ptr, const char* func, const char* file, int line);
#define magma_free(ptr) magma_free_internal(ptr, __func__, __FILE__, __LINE__)
/* interface_cuda/alloc.cpp:242 (magma_malloc_pinned), :276 (magma_free_pinned_internal):
 * page-locked host memory, MAGMA_ERR_HOST_ALLOC / MAGMA_ERR_INVALID_PTR on failure */
magma_int_t magma_malloc_pinned(void** ptr_ptr, size_t bytes);
magma_int_t magma_free_pinned_internal(void* ptr, const char* func, const char* file, int line);
#define magma_free_pinned(ptr) magma_free_pinned_internal(ptr, __func__, __FILE__, __LINE__)

/* include/magma_auxiliary.h:248-281 (queue support; the public names are
 * macros over the *_internal symbols, exactly as in MAGMA). */
void magma_queue_create_internal(magma_device_t device, magma_queue_t* queue_ptr,
                                 const char* func, const char* file, int line);
void magma_queue_create_from_cuda_internal(magma_device_t device, cudaStream_t stream,
                                           cublasHandle_t cublas, cusparseHandle_t cusparse,
                                           magma_queue_t* queue_ptr,
                                           const char* func, const char* file, int line);
void magma_queue_destroy_internal(magma_queue_t queue, const char* func, const char* file, int line);
void magma_queue_sync_internal(magma_queue_t queue, const char* func, const char* file, int line);
magma_int_t  magma_queue_get_device(magma_queue_t queue);
cudaStream_t magma_queue_get_cuda_stream(magma_queue_t queue);

/* No reference counterpart (MAGMA allocates workspace inside every call,
 * src/zgetrf_batched.cpp:148-170). Reserves at least `bytes` of the queue's
 * grow-only device workspace now, so that later calls never allocate -- call
 * it before capturing batched calls into a CUDA graph. */
magma_int_t  magma_queue_reserve_workspace(magma_queue_t queue, size_t bytes);

/* No reference counterpart. Caps the queue's device workspace at `bytes` (a
 * workspace already larger is freed after the queue's stream drains). A call that
 * would need more returns MAGMA_ERR_DEVICE_ALLOC before enqueueing any work, as
 * the reference does when its per-call cudaMalloc fails (src/zgetrf_batched.cpp:
 * 172-194, src/zpotrf_vbatched.cpp:99,124). For callers with a fixed device-memory
 * budget. Returns MAGMA_SUCCESS, or -1 for a null queue. */
magma_int_t  magma_b200_queue_set_workspace_limit(magma_queue_t queue, size_t bytes);

/* No reference counterpart (the reference's timers are host wall clocks around
 * whole calls). With stage timing on, multi-kernel routines record CUDA events
 * on the queue's stream at their stage boundaries -- magma_dgesv_batched
 * (n > 64): getrf, getrs; magma_dsgesv_batched: LU, refinement, FP64 fallback --
 * and magma_b200_stage_times returns the last such call's stage durations in ms
 * (waits for its last event; returns the number of stages written, <= max). */
magma_int_t  magma_b200_stage_timing(magma_queue_t queue, magma_int_t enable);
magma_int_t  magma_b200_stage_times(magma_queue_t queue, float* ms, magma_int_t max);

/* No reference counterpart; a test hook. With cycles > 0, the tensor-core LU of
 * magma_dsgesv_batched issues no tensor-core work and bounds each completion wait
 * at `cycles` clock cycles, so the first wait runs out with nothing in flight: the
 * kernel raises its error flag, releases its tensor memory and hands its instances
 * to the FP64 fallback (iter -3), the path a real time-out takes. 0 restores normal
 * operation. Process-wide; for tests only. */
void magma_b200_debug_tc_wait_limit(long long cycles);

#define magma_queue_create(device, queue_ptr) \
        magma_queue_create_internal(device, queue_ptr, __func__, __FILE__, __LINE__)
#define magma_queue_create_from_cuda(device, stream, cublas, cusparse, queue_ptr) \
        magma_queue_create_from_cuda_internal(device, stream, cublas, cusparse, queue_ptr, __func__, __FILE__, __LINE__)
#define magma_queue_destroy(queue) magma_queue_destroy_internal(queue, __func__, __FILE__, __LINE__)
#define magma_queue_sync(queue)    magma_queue_sync_internal(queue, __func__, __FILE__, __LINE__)

/* include/magma_copy.h:45-84 (setvector / getvector, sync and async) */
void magma_setvector_internal(magma_int_t n, magma_int_t elemSize, const void* hx_src, magma_int_t incx,
                              magma_ptr dy_dst, magma_int_t incy, magma_queue_t queue,
                              const char* func, const char* file, int line);
void magma_getvector_internal(magma_int_t n, magma_int_t elemSize, const void* dx_src, magma_int_t incx,
                              void* hy_dst, magma_int_t incy, magma_queue_t queue,
                              const char* func, const char* file, int line);
void magma_setvector_async_internal(magma_int_t n, magma_int_t elemSize, const void* hx_src, magma_int_t incx,
                                    magma_ptr dy_dst, magma_int_t incy, magma_queue_t queue,
                                    const char* func, const char* file, int line);
void magma_getvector_async_internal(magma_int_t n, magma_int_t elemSize, const void* dx_src, magma_int_t incx,
                                    void* hy_dst, magma_int_t incy, magma_queue_t queue,
                                    const char* func, const char* file, int line);
#define magma_setvector(n, es, hx, incx, dy, incy, queue) \
        magma_setvector_internal(n, es, hx, incx, dy, incy, queue, __func__, __FILE__, __LINE__)
#define magma_getvector(n, es, dx, incx, hy, incy, queue) \
        magma_getvector_internal(n, es, dx, incx, hy, incy, queue, __func__, __FILE__, __LINE__)
#define magma_setvector_async(n, es, hx, incx, dy, incy, queue) \
        magma_setvector_async_internal(n, es, hx, incx, dy, incy, queue, __func__, __FILE__, __LINE__)
#define magma_getvector_async(n, es, dx, incx, hy, incy, queue) \
        magma_getvector_async_internal(n, es, dx, incx, hy, incy, queue, __func__, __FILE__, __LINE__)

/* Pointer-array builders: output_array[i] = input + (batch_offset*i) + row + column*lda.
 * magmablas/zset_pointer.cu:17-26 (kernel), :87 (magma_zset_pointer);
 * magmablas/set_pointer.cu:72 (magma_iset_pointer). One launch, no host round trip. */
void magma_dset_pointer(double** output_array, double* input, magma_int_t lda,
                        magma_int_t row, magma_int_t column, magma_int_t batch_offset,
                        magma_int_t batchCount, magma_queue_t queue);
void magma_sset_pointer(float** output_array, float* input, magma_int_t lda,
                        magma_int_t row, magma_int_t column, magma_int_t batch_offset,
                        magma_int_t batchCount, magma_queue_t queue);
void magma_iset_pointer(magma_int_t** output_array, magma_int_t* input, magma_int_t lda,
                        magma_int_t row, magma_int_t column, magma_int_t batch_offset,
                        magma_int_t batchCount, magma_queue_t queue);

/* ------------------------------------------------------------------------
 * Batched LU (fixed size)
 * ---------------------------------------------------------------------- */

/* P*A = L*U with partial pivoting (ties -> lowest row, as LAPACK idamax).
 * src/zgetrf_batched.cpp:83-89; arg checks :96-107 (m:-1, n:-2, ldda:-4). */
magma_int_t magma_dgetrf_batched(magma_int_t m, magma_int_t n, double** dA_array, magma_int_t ldda,
                                 magma_int_t** ipiv_array, magma_int_t* info_array,
                                 magma_int_t batchCount, magma_queue_t queue);

/* Solve op(A) X = B with the factors of magma_dgetrf_batched.
 * src/zgetrs_batched.cpp:87-118 (trans:-1, n:-2, nrhs:-3, ldda:-5, lddb:-8). */
magma_int_t magma_dgetrs_batched(magma_trans_t trans, magma_int_t n, magma_int_t nrhs,
                                 double** dA_array, magma_int_t ldda, magma_int_t** dipiv_array,
                                 double** dB_array, magma_int_t lddb,
                                 magma_int_t batchCount, magma_queue_t queue);

/* getrf + getrs. src/zgesv_batched.cpp:93-147 (n:-1, nrhs:-2, ldda:-4, lddb:-6). */
magma_int_t magma_dgesv_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                magma_int_t** dipiv_array, double** dB_array, magma_int_t lddb,
                                magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue);


/* Variable-size batched LU. No counterpart in MAGMA 2.2 (its only vbatched
 * LAPACK routine is potrf, include/magma_zvbatched.h:29-70); defined by analogy
 * with magma_dpotrf_vbatched: m, n, nrhs, ldda, lddb are device arrays of
 * batchCount+1 entries; checked forms reduce the sizes on the device (one host
 * synchronisation), _max_nocheck forms take the maxima and never synchronise.
 * max(m, n) <= 1024. Pivots, info and factors as magma_dgetrf_batched.
 * Checks: getrf m -1, n -2, ldda -4, batchCount -7; getrs trans -1, n -2,
 * nrhs -3, ldda -5, lddb -8, batchCount -10; gesv n -1, nrhs -2, ldda -4,
 * lddb -7, batchCount -9. */
magma_int_t magma_dgetrf_vbatched(magma_int_t* m, magma_int_t* n, double** dA_array, magma_int_t* ldda,
                                  magma_int_t** ipiv_array, magma_int_t* info_array, magma_int_t batchCount,
                                  magma_queue_t queue);
magma_int_t magma_dgetrf_vbatched_max_nocheck(magma_int_t* m, magma_int_t* n, double** dA_array, magma_int_t* ldda,
                                              magma_int_t** ipiv_array, magma_int_t* info_array,
                                              magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                              magma_queue_t queue);
magma_int_t magma_dgetrs_vbatched(magma_trans_t trans, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                  magma_int_t* ldda, magma_int_t** dipiv_array, double** dB_array, magma_int_t* lddb,
                                  magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_dgetrs_vbatched_max_nocheck(magma_trans_t trans, magma_int_t* n, magma_int_t* nrhs,
                                              double** dA_array, magma_int_t* ldda, magma_int_t** dipiv_array,
                                              double** dB_array, magma_int_t* lddb, magma_int_t batchCount,
                                              magma_int_t max_n, magma_int_t max_nrhs, magma_queue_t queue);
magma_int_t magma_dgesv_vbatched(magma_int_t* n, magma_int_t* nrhs, double** dA_array, magma_int_t* ldda,
                                 magma_int_t** dipiv_array, double** dB_array, magma_int_t* lddb,
                                 magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_dgesv_vbatched_max_nocheck(magma_int_t* n, magma_int_t* nrhs, double** dA_array, magma_int_t* ldda,
                                             magma_int_t** dipiv_array, double** dB_array, magma_int_t* lddb,
                                             magma_int_t* dinfo_array, magma_int_t batchCount, magma_int_t max_n,
                                             magma_int_t max_nrhs, magma_queue_t queue);

/* Single-precision forms (generated from the same templates in MAGMA:
 * src/zgetrf_batched.cpp:83, src/zgetrs_batched.cpp:87, src/zgesv_batched.cpp:93). */
magma_int_t magma_sgetrf_batched(magma_int_t m, magma_int_t n, float** dA_array, magma_int_t ldda,
                                 magma_int_t** ipiv_array, magma_int_t* info_array, magma_int_t batchCount,
                                 magma_queue_t queue);
magma_int_t magma_sgetrs_batched(magma_trans_t trans, magma_int_t n, magma_int_t nrhs, float** dA_array,
                                 magma_int_t ldda, magma_int_t** dipiv_array, float** dB_array, magma_int_t lddb,
                                 magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_sgesv_batched(magma_int_t n, magma_int_t nrhs, float** dA_array, magma_int_t ldda,
                                magma_int_t** dipiv_array, float** dB_array, magma_int_t lddb,
                                magma_int_t* dinfo_array, magma_int_t batchCount, magma_queue_t queue);

/* LU without pivoting and its solves: src/zgetrf_nopiv_batched.cpp:76-94 (m -1, n -2,
 * ldda -4), src/zgetrs_nopiv_batched.cpp:89-113 (trans -1, n -2, nrhs -3, ldda -5,
 * lddb -8; info_array set to 0), src/zgesv_nopiv_batched.cpp:87-104 (n -1, nrhs -2,
 * ldda -4, lddb -6). info_array: first zero pivot (1-based); a zero pivot is not
 * divided by. Same kernels (and sizes) as the pivoted forms. */
magma_int_t magma_dgetrf_nopiv_batched(magma_int_t m, magma_int_t n, double** dA_array, magma_int_t ldda,
                                       magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_dgetrs_nopiv_batched(magma_trans_t trans, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                       magma_int_t ldda, double** dB_array, magma_int_t lddb,
                                       magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_dgesv_nopiv_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                      double** dB_array, magma_int_t lddb, magma_int_t* info_array,
                                      magma_int_t batchCount, magma_queue_t queue);

/* Random butterfly transformation (src/zgerbt_batched.cpp:118-190; checks gen -1,
 * n -2, nrhs -3, ldda -5, lddb -7, also stored in *info): A_i <- U^T A_i V,
 * B_i <- U^T B_i with the depth-2 butterflies built from the HOST vectors U and V
 * (2n entries each; filled from a fixed-seed generator when gen is MagmaTrue).
 * magma_dgesv_rbt_batched (src/zgesv_rbt_batched.cpp:81-170; n -1, nrhs -2,
 * ldda -4, lddb -6): transform, LU without pivoting, solve, x = V y.
 * n must be a multiple of 4 (MAGMA_ERR_NOT_SUPPORTED otherwise), n <= 1024. */
magma_int_t magma_dgerbt_batched(magma_bool_t gen, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                 magma_int_t ldda, double** dB_array, magma_int_t lddb, double* U, double* V,
                                 magma_int_t* info, magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_dgesv_rbt_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                    double** dB_array, magma_int_t lddb, magma_int_t* dinfo_array,
                                    magma_int_t batchCount, magma_queue_t queue);

/* Householder QR: src/zgeqrf_batched.cpp:89-119 (info_array zeroed first; m -1, n -2,
 * ldda -4). LAPACK's representation: R on and above the diagonal, the reflectors'
 * vectors below it (unit leading entry implied), tau_i (min(m,n) entries) per
 * instance. m <= 1024 (MAGMA_ERR_NOT_SUPPORTED otherwise), any n. */
magma_int_t magma_dgeqrf_batched(magma_int_t m, magma_int_t n, double** dA_array, magma_int_t ldda,
                                 double** dtau_array, magma_int_t* info_array, magma_int_t batchCount,
                                 magma_queue_t queue);

/* Inverse from the getrf factors into a separate array: dinvA_i = inv(A_i).
 * src/zgetri_outofplace_batched.cpp:82-220; checks n -1, ldda -3, lddia -6.
 * info_array (may be NULL): 1-based index of the first exactly-zero U(i,i), else 0.
 * Each column of the result is bit-identical to getrs applied to the matching
 * unit vector. n <= 1024. */
magma_int_t magma_dgetri_outofplace_batched(magma_int_t n, double** dA_array, magma_int_t ldda,
                                            magma_int_t** dipiv_array, double** dinvA_array, magma_int_t lddia,
                                            magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue);

/* Mixed precision: FP32 LU + FP64 iterative refinement with FP64 fallback.
 * No batched counterpart in MAGMA 2.2; per instance it is magma_dsgesv_gpu
 * (src/zcgesv_gpu.cpp:144-365): stopping test max|R_j| <= max|X_j| ||A||_inf
 * eps sqrt(n), ITERMAX 30. iter_array[i]: >= 0 iterations used; -2 overflow in
 * the conversion to single; -3 singular in single; -31 no convergence (also
 * reported early when the residual stops halving). Negative iter means the
 * instance was re-solved in double (A then holds the double LU factors and
 * ipiv the double pivots; info its getrf info). Checks: n -1, nrhs -2,
 * ldda -4, lddb -7, lddx -9. B is not modified. n <= 512. */
magma_int_t magma_dsgesv_batched(magma_int_t n, magma_int_t nrhs, double** dA_array, magma_int_t ldda,
                                 magma_int_t** dipiv_array, double** dB_array, magma_int_t lddb, double** dX_array,
                                 magma_int_t lddx, magma_int_t* iter_array, magma_int_t* dinfo_array,
                                 magma_int_t batchCount, magma_queue_t queue);

/* Mixed-precision Cholesky solve on variable sizes: FP32 potrf + FP64 refinement
 * with FP64 fallback. No batched counterpart in MAGMA 2.2; per instance it is
 * magma_dsposv_gpu (src/zcposv_gpu.cpp:134-330) with the vbatched conventions of
 * magma_dpotrf_vbatched (include/magma_zvbatched.h:59-70): device size arrays of
 * batchCount+1 entries and, like the reference's variable-size Cholesky, uplo =
 * MagmaLower only (MagmaUpper returns MAGMA_ERR_NOT_SUPPORTED). dworks_array[i]
 * is caller-owned single-precision workspace of at least n_i*(n_i+nrhs_i)
 * floats (the reference's dworks). iter_array / info_array as
 * magma_dsgesv_batched (info: dpotrf info of the FP64 fallback). Checks: uplo
 * -1, n -2, nrhs -3, ldda -5, lddb -7, lddx -9, batchCount -13. max_n <= 512. */
magma_int_t magma_dsposv_vbatched(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                  magma_int_t* ldda, double** dB_array, magma_int_t* lddb, double** dX_array,
                                  magma_int_t* lddx, float** dworks_array, magma_int_t* iter_array,
                                  magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_dsposv_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs,
                                              double** dA_array, magma_int_t* ldda, double** dB_array,
                                              magma_int_t* lddb, double** dX_array, magma_int_t* lddx,
                                              float** dworks_array, magma_int_t* iter_array,
                                              magma_int_t* info_array, magma_int_t batchCount, magma_int_t max_n,
                                              magma_int_t max_nrhs, magma_queue_t queue);

/* ------------------------------------------------------------------------
 * Batched Cholesky (fixed size). Lower and Upper are both supported (the
 * reference's batched potrf handles Lower only, src/zpotf2_vbatched.cpp:32-34).
 * ---------------------------------------------------------------------- */

/* A = L L^T (or U^T U). src/zpotrf_batched.cpp:291-320: info zeroed first;
 * uplo -1, n -2, ldda -4. info_array[i] = order of the first non-positive
 * (or NaN) leading minor, as LAPACK dpotrf. */
magma_int_t magma_dpotrf_batched(magma_uplo_t uplo, magma_int_t n, double** dA_array, magma_int_t ldda,
                                 magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue);

/* src/zpotrs_batched.cpp:71-94 (last failing argument wins: uplo -1, n -2,
 * nrhs -3, ldda -5, lddb -7). */
magma_int_t magma_dpotrs_batched(magma_uplo_t uplo, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                 magma_int_t ldda, double** dB_array, magma_int_t lddb, magma_int_t batchCount,
                                 magma_queue_t queue);

/* potrf + potrs. src/zposv_batched.cpp:89-141. */
magma_int_t magma_dposv_batched(magma_uplo_t uplo, magma_int_t n, magma_int_t nrhs, double** dA_array,
                                magma_int_t ldda, double** dB_array, magma_int_t lddb, magma_int_t* dinfo_array,
                                magma_int_t batchCount, magma_queue_t queue);

/* ------------------------------------------------------------------------
 * Variable-size batched Cholesky. n, nrhs, ldda, lddb are device arrays of
 * batchCount+1 entries. The checked forms reduce the sizes on the device and
 * read the maxima back (one host synchronisation, as the reference);
 * _max_nocheck forms take the maxima from the caller and never synchronise.
 * ---------------------------------------------------------------------- */

/* include/magma_zvbatched.h:66-70, src/zpotrf_vbatched.cpp:335-356; checks as
 * magmablas/vbatched_check.cu:840-892 (uplo -1, n -2, ldda -4, batchCount -6). */
magma_int_t magma_dpotrf_vbatched(magma_uplo_t uplo, magma_int_t* n, double** dA_array, magma_int_t* ldda,
                                  magma_int_t* info_array, magma_int_t batchCount, magma_queue_t queue);
/* include/magma_zvbatched.h:59-64, src/zpotrf_vbatched.cpp:251-267. */
magma_int_t magma_dpotrf_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, double** dA_array,
                                              magma_int_t* ldda, magma_int_t* info_array, magma_int_t batchCount,
                                              magma_int_t max_n, magma_queue_t queue);

/* No counterpart in the reference. Same contract and results as
 * magma_dpotrf_vbatched_max_nocheck, for callers that cannot allocate device
 * memory (a stream being captured into a CUDA graph, a fixed device-memory
 * budget, allocator callbacks): its scratch is a static device array built
 * into the library (about 2 MiB per GPU that loads it, held until exit)
 * instead of queue workspace. At most 65536 instances per call; larger
 * batches return -6 with a message. The first call on a device looks up the
 * array's address (cudaGetSymbolAddress), so make it before any stream
 * capture. All calls share the array: calls whose work can overlap on the
 * GPU (unordered streams) race and must be serialised by the caller. */
magma_int_t magma_dpotrf_vbatched_max_nocheck_noalloc(magma_uplo_t uplo, magma_int_t* n, double** dA_array,
                                                      magma_int_t* ldda, magma_int_t* info_array,
                                                      magma_int_t batchCount, magma_int_t max_n,
                                                      magma_queue_t queue);

/* No counterpart in MAGMA 2.2 (potrs is fixed-size only, src/zpotrs_batched.cpp:71);
 * defined by analogy with magma_dpotrf_vbatched. Checks: uplo -1, n -2, nrhs -3,
 * ldda -5, lddb -7, batchCount -9. */
magma_int_t magma_dpotrs_vbatched(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                  magma_int_t* ldda, double** dB_array, magma_int_t* lddb, magma_int_t batchCount,
                                  magma_queue_t queue);
magma_int_t magma_dpotrs_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs,
                                              double** dA_array, magma_int_t* ldda, double** dB_array,
                                              magma_int_t* lddb, magma_int_t batchCount, magma_int_t max_n,
                                              magma_int_t max_nrhs, magma_queue_t queue);

/* No counterpart in MAGMA 2.2: potrf + potrs on variable sizes (checks as potrs,
 * batchCount -10). */
magma_int_t magma_dposv_vbatched(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs, double** dA_array,
                                 magma_int_t* ldda, double** dB_array, magma_int_t* lddb, magma_int_t* dinfo_array,
                                 magma_int_t batchCount, magma_queue_t queue);
magma_int_t magma_dposv_vbatched_max_nocheck(magma_uplo_t uplo, magma_int_t* n, magma_int_t* nrhs,
                                             double** dA_array, magma_int_t* ldda, double** dB_array,
                                             magma_int_t* lddb, magma_int_t* dinfo_array, magma_int_t batchCount,
                                             magma_int_t max_n, magma_int_t max_nrhs, magma_queue_t queue);

/* ------------------------------------------------------------------------
 * Systems in host memory (no reference counterpart: MAGMA's batched routines take
 * device pointer arrays only, and its testers upload, solve and read back in
 * sequence, testing/testing_zgesv_batched.cpp:111-125). A solver owns device
 * staging buffers, pointer arrays, two copy streams and per-chunk events for
 * `batch` systems of order n with nrhs right-hand sides, cut into `chunks` chunks;
 * magma_b200_host_solve queues every chunk's upload on one copy stream, solves each
 * chunk on the queue's stream as soon as it has landed (magma_dsgesv_batched for
 * MAGMA_B200_HOST_DSGESV, magma_dgesv_batched for MAGMA_B200_HOST_DGESV) and reads its
 * results back on a second copy stream, so transfers overlap the solves. Host layouts
 * are packed batches of column-major matrices: hA batch x (n x lda), hB batch x
 * (n x nrhs, ldb); outputs hX (DSGESV: batch x (n x nrhs, ld n); DGESV: the solutions
 * in hB's layout), hI (DSGESV: iter per system; DGESV: batch x n pivots) and hInfo
 * (batch). A solve returns once everything is queued (the first solver error, or
 * MAGMA_SUCCESS); synchronising the queue covers the whole sequence. Page-locked
 * host memory is needed for the copies to overlap (pageable memory gives the same
 * results in sequence). create returns -1..-9 for an illegal argument or
 * MAGMA_ERR_DEVICE_ALLOC; chunk_start returns chunk c's first system (c = chunks:
 * batch), -1 out of range. */
enum { MAGMA_B200_HOST_DSGESV = 0, MAGMA_B200_HOST_DGESV = 1 };
struct magma_b200_host_solver;
typedef struct magma_b200_host_solver* magma_b200_host_solver_t;
magma_int_t magma_b200_host_solver_create(magma_int_t kind, magma_int_t batch, magma_int_t n, magma_int_t nrhs,
                                          magma_int_t lda, magma_int_t ldb, magma_int_t chunks, magma_queue_t queue,
                                          magma_b200_host_solver_t* solver);
magma_int_t magma_b200_host_solve(magma_b200_host_solver_t solver, const double* hA, const double* hB, double* hX,
                                  magma_int_t* hI, magma_int_t* hInfo);
magma_int_t magma_b200_host_solver_chunk_start(magma_b200_host_solver_t solver, magma_int_t c);
magma_int_t magma_b200_host_solver_destroy(magma_b200_host_solver_t solver);

/* ------------------------------------------------------------------------
 * Kernel-variant tuning (no reference counterpart; takes the role of the
 * reference's static tables control/batched_kernel_param.h and the headers
 * under magmablas/gemm_config/). The table holds 21 values: the GEMM tile variant
 * (0: 64x64, 1: 32x32, 2: 16x16; 3: on the tensor cores, FP64 64x64 with mma.sync
 * .f64 (bit-identical to 0-2) and FP32 128x128 with tcgen05 split TF32 (within the
 * reference tester's 30 eps bound, not bit-identical to 0-2)) for
 * max(M,N) <= 16, <= 32, <= 64 and larger, first for FP64 then FP32; 1/0 for the
 * tensor-core LU in magma_dsgesv_batched (n = 96..256, step 32) as a whole; 1/0 for
 * the FP64 blocked LU's trailing update on the tensor cores (DMMA) instead of the
 * FP64 pipe, for max(m) <= 128, <= 256, <= 512, <= 1024; and 1/0 for the tensor-core
 * LU (with its fused refinement) at each order n = 96, 128, ..., 256; 1/0 for the
 * variable-size FP64 Cholesky (potrf / potrs / posv vbatched) as one persistent
 * launch over all orders <= 512 instead of one launch per size bucket; and 1/0 for
 * the same choice in the variable-size FP64 LU (getrf / gesv vbatched). Tables of 9,
 * 13, 19 or 20 values (saved before the later entries existed) are accepted and leave
 * the rest unchanged. Defaults are built in;
 * MAGMA_B200_TUNING=<file> loads a saved table at first use. Variants of one
 * family compute bit-identical results (except the FP32 tensor-core tile, noted above);
 * tuning changes speed only. Not to be
 * called while other calls of this library are in flight.
 * magma_b200_autotune times every variant on the queue's device with synthetic
 * problems and keeps the fastest (synchronises the queue). tuning_get returns
 * the number of values (21) and fills `values` when count >= 21; tuning_set
 * returns MAGMA_ERR_ILLEGAL_VALUE for a wrong count or an out-of-range value. */
magma_int_t magma_b200_autotune(magma_queue_t queue);
magma_int_t magma_b200_tuning_get(magma_int_t* values, magma_int_t count);
magma_int_t magma_b200_tuning_set(const magma_int_t* values, magma_int_t count);
magma_int_t magma_b200_tuning_save(const char* path);
magma_int_t magma_b200_tuning_load(const char* path);

/* ------------------------------------------------------------------------
 * Batched GEMM: C_i = alpha op(A_i) op(B_i) + beta C_i (C not read when beta == 0,
 * magmablas/gemm_template_device.cuh:197). Checks as
 * magmablas/dgemm_batched_core.cu:180-213 (transA -1, transB -2, m -3, n -4, k -5,
 * ldda -8, lddb -10, lddc -13; quick return when m, n or k <= 0).
 * ---------------------------------------------------------------------- */
/* magmablas/zgemm_batched.cpp:148-160 */
void magmablas_dgemm_batched(magma_trans_t transA, magma_trans_t transB, magma_int_t m, magma_int_t n, magma_int_t k,
                             double alpha, double const* const* dA_array, magma_int_t ldda,
                             double const* const* dB_array, magma_int_t lddb, double beta, double** dC_array,
                             magma_int_t lddc, magma_int_t batchCount, magma_queue_t queue);
/* magmablas/zgemm_batched.cpp:169-196 (the reference picks cuBLAS or its own kernel; here always the library's) */
void magma_dgemm_batched(magma_trans_t transA, magma_trans_t transB, magma_int_t m, magma_int_t n, magma_int_t k,
                         double alpha, double const* const* dA_array, magma_int_t ldda, double const* const* dB_array,
                         magma_int_t lddb, double beta, double** dC_array, magma_int_t lddc, magma_int_t batchCount,
                         magma_queue_t queue);
void magmablas_sgemm_batched(magma_trans_t transA, magma_trans_t transB, magma_int_t m, magma_int_t n, magma_int_t k,
                             float alpha, float const* const* dA_array, magma_int_t ldda, float const* const* dB_array,
                             magma_int_t lddb, float beta, float** dC_array, magma_int_t lddc, magma_int_t batchCount,
                             magma_queue_t queue);
void magma_sgemm_batched(magma_trans_t transA, magma_trans_t transB, magma_int_t m, magma_int_t n, magma_int_t k,
                         float alpha, float const* const* dA_array, magma_int_t ldda, float const* const* dB_array,
                         magma_int_t lddb, float beta, float** dC_array, magma_int_t lddc, magma_int_t batchCount,
                         magma_queue_t queue);

/* Variable-size GEMM, m/n/k/ldda/lddb/lddc device arrays of batchCount+1 entries.
 * magmablas/zgemm_vbatched.cpp:235-271 (checked; one host synchronisation for the
 * checker and the maxima), :19-29 (_max_nocheck), :33 (_max), :81 (_nocheck);
 * checks as magmablas/vbatched_check.cu:78-99 (batchCount -14).
 * Argument order of _max_nocheck and _max: (..., lddc, batchCount, max_m, max_n, max_k,
 * queue), as the reference DEFINES them (magmablas/zgemm_vbatched.cpp:19-29, 46-56) and as
 * every caller inside the reference passes them (magmablas/ztrsm_vbatched_core.cu:235-236,
 * zgemm_vbatched.cpp:99-106, testing/testing_zgemm_vbatched.cpp:244-251). The reference's
 * public header declares (max_m, max_n, max_k, batchCount) instead
 * (include/magma_zvbatched.h:90-112); the four are all magma_int_t, so the reference reads
 * them in definition order whatever a caller compiled against, and so does this library. */
void magmablas_dgemm_vbatched(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                              magma_int_t* k, double alpha, double const* const* dA_array, magma_int_t* ldda,
                              double const* const* dB_array, magma_int_t* lddb, double beta, double** dC_array,
                              magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue);
void magmablas_dgemm_vbatched_max_nocheck(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                                          magma_int_t* k, double alpha, double const* const* dA_array,
                                          magma_int_t* ldda, double const* const* dB_array, magma_int_t* lddb,
                                          double beta, double** dC_array, magma_int_t* lddc, magma_int_t batchCount,
                                          magma_int_t max_m, magma_int_t max_n, magma_int_t max_k,
                                          magma_queue_t queue);
void magmablas_dgemm_vbatched_max(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                                  magma_int_t* k, double alpha, double const* const* dA_array, magma_int_t* ldda,
                                  double const* const* dB_array, magma_int_t* lddb, double beta, double** dC_array,
                                  magma_int_t* lddc, magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                  magma_int_t max_k, magma_queue_t queue);
void magmablas_dgemm_vbatched_nocheck(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                                      magma_int_t* k, double alpha, double const* const* dA_array, magma_int_t* ldda,
                                      double const* const* dB_array, magma_int_t* lddb, double beta,
                                      double** dC_array, magma_int_t* lddc, magma_int_t batchCount,
                                      magma_queue_t queue);
void magmablas_sgemm_vbatched(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                              magma_int_t* k, float alpha, float const* const* dA_array, magma_int_t* ldda,
                              float const* const* dB_array, magma_int_t* lddb, float beta, float** dC_array,
                              magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue);
void magmablas_sgemm_vbatched_max_nocheck(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                                          magma_int_t* k, float alpha, float const* const* dA_array,
                                          magma_int_t* ldda, float const* const* dB_array, magma_int_t* lddb,
                                          float beta, float** dC_array, magma_int_t* lddc, magma_int_t batchCount,
                                          magma_int_t max_m, magma_int_t max_n, magma_int_t max_k,
                                          magma_queue_t queue);
void magmablas_sgemm_vbatched_max(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                                  magma_int_t* k, float alpha, float const* const* dA_array, magma_int_t* ldda,
                                  float const* const* dB_array, magma_int_t* lddb, float beta, float** dC_array,
                                  magma_int_t* lddc, magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                  magma_int_t max_k, magma_queue_t queue);
void magmablas_sgemm_vbatched_nocheck(magma_trans_t transA, magma_trans_t transB, magma_int_t* m, magma_int_t* n,
                                      magma_int_t* k, float alpha, float const* const* dA_array, magma_int_t* ldda,
                                      float const* const* dB_array, magma_int_t* lddb, float beta, float** dC_array,
                                      magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue);

/* Variable-size SYRK on one triangle: C = alpha op(A) op(A)^T + beta C (uplo part only).
 * include/magma_zvbatched.h:202-243, magmablas/zsyrk_vbatched.cpp; checks as
 * magmablas/vbatched_check.cu:186-262 (uplo -1, trans -2, n -3, k -4, ldda -7,
 * lddc -10, batchCount -11). n, k, ldda, lddc: device arrays of batchCount+1 entries. */
void magmablas_dsyrk_vbatched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k, double alpha,
                              double const* const* dA_array, magma_int_t* ldda, double beta, double** dC_array,
                              magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue);
void magmablas_dsyrk_vbatched_max_nocheck(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,
                                          double alpha, double const* const* dA_array, magma_int_t* ldda,
                                          double beta, double** dC_array, magma_int_t* lddc, magma_int_t batchCount,
                                          magma_int_t max_n, magma_int_t max_k, magma_queue_t queue);
void magmablas_dsyrk_vbatched_max(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,
                                  double alpha, double const* const* dA_array, magma_int_t* ldda, double beta,
                                  double** dC_array, magma_int_t* lddc, magma_int_t batchCount, magma_int_t max_n,
                                  magma_int_t max_k, magma_queue_t queue);
void magmablas_dsyrk_vbatched_nocheck(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,
                                      double alpha, double const* const* dA_array, magma_int_t* ldda, double beta,
                                      double** dC_array, magma_int_t* lddc, magma_int_t batchCount,
                                      magma_queue_t queue);
void magmablas_ssyrk_vbatched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k, float alpha,
                              float const* const* dA_array, magma_int_t* ldda, float beta, float** dC_array,
                              magma_int_t* lddc, magma_int_t batchCount, magma_queue_t queue);
void magmablas_ssyrk_vbatched_max_nocheck(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,
                                          float alpha, float const* const* dA_array, magma_int_t* ldda, float beta,
                                          float** dC_array, magma_int_t* lddc, magma_int_t batchCount,
                                          magma_int_t max_n, magma_int_t max_k, magma_queue_t queue);
void magmablas_ssyrk_vbatched_max(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,
                                  float alpha, float const* const* dA_array, magma_int_t* ldda, float beta,
                                  float** dC_array, magma_int_t* lddc, magma_int_t batchCount, magma_int_t max_n,
                                  magma_int_t max_k, magma_queue_t queue);
void magmablas_ssyrk_vbatched_nocheck(magma_uplo_t uplo, magma_trans_t trans, magma_int_t* n, magma_int_t* k,
                                      float alpha, float const* const* dA_array, magma_int_t* ldda, float beta,
                                      float** dC_array, magma_int_t* lddc, magma_int_t batchCount,
                                      magma_queue_t queue);

/* Variable-size triangular solve op(A) X = alpha B / X op(A) = alpha B (X overwrites B)
 * and triangular multiply B = alpha op(A) B / alpha B op(A).
 * include/magma_zvbatched.h:324-450, magmablas/ztrsm_vbatched.cpp:21-215,
 * magmablas/ztrmm_vbatched.cpp:21-90; checks as magmablas/vbatched_check.cu:134-181 and
 * :785-833 (side -1, uplo -2, transA -3, diag -4, m -5, n -6, ldda -9, lddb -11,
 * batchCount -12). m, n, ldda, lddb: device arrays of batchCount+1 entries. */
void magmablas_dtrsm_vbatched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                              magma_int_t* m, magma_int_t* n, double alpha, double** dA_array, magma_int_t* ldda,
                              double** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_queue_t queue);
void magmablas_dtrsm_vbatched_max_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,
                                          magma_diag_t diag, magma_int_t* m, magma_int_t* n, double alpha,
                                          double** dA_array, magma_int_t* ldda, double** dB_array, magma_int_t* lddb,
                                          magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                          magma_queue_t queue);
void magmablas_dtrsm_vbatched_max(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                  magma_int_t* m, magma_int_t* n, double alpha, double** dA_array, magma_int_t* ldda,
                                  double** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_int_t max_m,
                                  magma_int_t max_n, magma_queue_t queue);
void magmablas_dtrsm_vbatched_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                      magma_int_t* m, magma_int_t* n, double alpha, double** dA_array,
                                      magma_int_t* ldda, double** dB_array, magma_int_t* lddb,
                                      magma_int_t batchCount, magma_queue_t queue);
void magmablas_strsm_vbatched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                              magma_int_t* m, magma_int_t* n, float alpha, float** dA_array, magma_int_t* ldda,
                              float** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_queue_t queue);
void magmablas_strsm_vbatched_max_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,
                                          magma_diag_t diag, magma_int_t* m, magma_int_t* n, float alpha,
                                          float** dA_array, magma_int_t* ldda, float** dB_array, magma_int_t* lddb,
                                          magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                          magma_queue_t queue);
void magmablas_strsm_vbatched_max(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                  magma_int_t* m, magma_int_t* n, float alpha, float** dA_array, magma_int_t* ldda,
                                  float** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_int_t max_m,
                                  magma_int_t max_n, magma_queue_t queue);
void magmablas_strsm_vbatched_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                      magma_int_t* m, magma_int_t* n, float alpha, float** dA_array,
                                      magma_int_t* ldda, float** dB_array, magma_int_t* lddb, magma_int_t batchCount,
                                      magma_queue_t queue);
void magmablas_dtrmm_vbatched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                              magma_int_t* m, magma_int_t* n, double alpha, double** dA_array, magma_int_t* ldda,
                              double** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_queue_t queue);
void magmablas_dtrmm_vbatched_max_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,
                                          magma_diag_t diag, magma_int_t* m, magma_int_t* n, double alpha,
                                          double** dA_array, magma_int_t* ldda, double** dB_array, magma_int_t* lddb,
                                          magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                          magma_queue_t queue);
void magmablas_dtrmm_vbatched_max(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                  magma_int_t* m, magma_int_t* n, double alpha, double** dA_array, magma_int_t* ldda,
                                  double** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_int_t max_m,
                                  magma_int_t max_n, magma_queue_t queue);
void magmablas_dtrmm_vbatched_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                      magma_int_t* m, magma_int_t* n, double alpha, double** dA_array,
                                      magma_int_t* ldda, double** dB_array, magma_int_t* lddb,
                                      magma_int_t batchCount, magma_queue_t queue);
void magmablas_strmm_vbatched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                              magma_int_t* m, magma_int_t* n, float alpha, float** dA_array, magma_int_t* ldda,
                              float** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_queue_t queue);
void magmablas_strmm_vbatched_max_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA,
                                          magma_diag_t diag, magma_int_t* m, magma_int_t* n, float alpha,
                                          float** dA_array, magma_int_t* ldda, float** dB_array, magma_int_t* lddb,
                                          magma_int_t batchCount, magma_int_t max_m, magma_int_t max_n,
                                          magma_queue_t queue);
void magmablas_strmm_vbatched_max(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                  magma_int_t* m, magma_int_t* n, float alpha, float** dA_array, magma_int_t* ldda,
                                  float** dB_array, magma_int_t* lddb, magma_int_t batchCount, magma_int_t max_m,
                                  magma_int_t max_n, magma_queue_t queue);
void magmablas_strmm_vbatched_nocheck(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                                      magma_int_t* m, magma_int_t* n, float alpha, float** dA_array,
                                      magma_int_t* ldda, float** dB_array, magma_int_t* lddb, magma_int_t batchCount,
                                      magma_queue_t queue);


/* Fixed-size forms (include/magma_zbatched.h:132-157,202-208,271-277): SYRK checks as
 * magmablas/zherk_batched_core.cu:233-258 (uplo -1, trans -2, n -3, k -4, ldda -7, lddc -10;
 * nothing done when n or k is 0); trsm/trmm as magmablas/ztrsm_batched.cpp:196-229 and
 * magmablas/ztrmm_batched_core.cu:811-832 (side -1, uplo -2, transA -3, diag -4, m -5, n -6,
 * ldda -9, lddb -11). The same kernels as the variable-size forms. */
void magmablas_dsyrk_batched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t n, magma_int_t k, double alpha,
                             double const* const* dA_array, magma_int_t ldda, double beta, double** dC_array,
                             magma_int_t lddc, magma_int_t batchCount, magma_queue_t queue);
void magma_dsyrk_batched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t n, magma_int_t k, double alpha,
                         double const* const* dA_array, magma_int_t ldda, double beta, double** dC_array,
                         magma_int_t lddc, magma_int_t batchCount, magma_queue_t queue);
void magmablas_dtrsm_batched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                             magma_int_t m, magma_int_t n, double alpha, double** dA_array, magma_int_t ldda,
                             double** dB_array, magma_int_t lddb, magma_int_t batchCount, magma_queue_t queue);
void magmablas_dtrmm_batched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                             magma_int_t m, magma_int_t n, double alpha, double** dA_array, magma_int_t ldda,
                             double** dB_array, magma_int_t lddb, magma_int_t batchCount, magma_queue_t queue);
void magmablas_ssyrk_batched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t n, magma_int_t k, float alpha,
                             float const* const* dA_array, magma_int_t ldda, float beta, float** dC_array,
                             magma_int_t lddc, magma_int_t batchCount, magma_queue_t queue);
void magma_ssyrk_batched(magma_uplo_t uplo, magma_trans_t trans, magma_int_t n, magma_int_t k, float alpha,
                         float const* const* dA_array, magma_int_t ldda, float beta, float** dC_array,
                         magma_int_t lddc, magma_int_t batchCount, magma_queue_t queue);
void magmablas_strsm_batched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                             magma_int_t m, magma_int_t n, float alpha, float** dA_array, magma_int_t ldda,
                             float** dB_array, magma_int_t lddb, magma_int_t batchCount, magma_queue_t queue);
void magmablas_strmm_batched(magma_side_t side, magma_uplo_t uplo, magma_trans_t transA, magma_diag_t diag,
                             magma_int_t m, magma_int_t n, float alpha, float** dA_array, magma_int_t ldda,
                             float** dB_array, magma_int_t lddb, magma_int_t batchCount, magma_queue_t queue);

#ifdef __cplusplus
}
#endif

#endif /* MAGMA_B200_H */
