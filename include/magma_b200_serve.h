/*
 * magma_b200_serve.h -- request loop for batched LU and Cholesky solves.
 *
 * No counterpart in the reference (MAGMA has no serving layer). The server
 * accepts solve requests of any size n <= 1024 and RHS count as they arrive
 * and runs them with continuous batching: whatever has been admitted while
 * earlier work was on the GPU goes out as the next micro-batch, on one of
 * several CUDA streams, so batches overlap on the device. With two or more
 * streams, requests of order n <= 128 and larger ones form separate batches on
 * separate streams, so small solves do not wait for large ones. Admission is by a
 * device-memory budget: a request waits (FIFO) until its matrix, right-hand
 * sides and pivots fit in the server's arena, and its memory is released when
 * its result has been copied back. Results are bit-identical to solving the
 * same request alone (each instance runs the same kernel whatever else is in
 * its batch).
 */
#ifndef MAGMA_B200_SERVE_H
#define MAGMA_B200_SERVE_H

#include "magma_b200_types.h"

#ifdef __cplusplus
extern "C" {
#endif

struct magma_b200_server;
typedef struct magma_b200_server* magma_b200_server_t;

enum { MAGMA_B200_SOLVE_LU = 0, MAGMA_B200_SOLVE_CHOLESKY = 1 };

/* Creates a server on `device` with a device arena of budget_bytes (one
 * cudaMalloc, here), `streams` CUDA streams (batches in flight) and at most
 * max_batch requests per micro-batch. Before returning it runs one small batch of
 * every kernel family and size bucket, so that no request pays a kernel's first-use
 * load. Each stream carries 4 auxiliary streams: the process should have
 * CUDA_DEVICE_MAX_CONNECTIONS >= 5 * streams (the library requests 32 at load time
 * unless it is already set). Returns MAGMA_SUCCESS or a MAGMA error. */
magma_int_t magma_b200_server_create(magma_int_t device, size_t budget_bytes, magma_int_t streams,
                                     magma_int_t max_batch, magma_b200_server_t* server);

/* Submits A X = B (kind LU, partial pivoting) or A X = B with A symmetric
 * positive definite (kind CHOLESKY, lower triangle used). A (n x n, lda),
 * B (n x nrhs, ldb) and X (n x nrhs, ldx) are column-major HOST buffers that
 * must stay valid and untouched until the request is reported complete;
 * page-locked buffers make the copies asynchronous. `tag` identifies the
 * request in magma_b200_server_poll. Returns MAGMA_SUCCESS, -1..-9 for an
 * illegal argument, or MAGMA_ERR_NOT_SUPPORTED when the request alone exceeds
 * the budget or n > 1024. */
magma_int_t magma_b200_server_submit(magma_b200_server_t server, magma_int_t kind, magma_int_t n, magma_int_t nrhs,
                                     const double* A, magma_int_t lda, const double* B, magma_int_t ldb, double* X,
                                     magma_int_t ldx, long long tag);

/* Reports up to `max` completed requests (each once): tag, info, submit and
 * completion times (steady clock, ns). info is LAPACK's (0, or > 0 for the first
 * zero pivot / non-positive minor), or a negative MAGMA error code when the solver
 * call of the request's batch failed. Returns the count. */
magma_int_t magma_b200_server_poll(magma_b200_server_t server, long long* tags, magma_int_t* infos,
                                   long long* t_submit_ns, long long* t_done_ns, magma_int_t max);

/* Caps the device workspace of each of the server's stream queues at `bytes`
 * (magma_b200_queue_set_workspace_limit; the workspace reserved at creation is
 * released when larger). Waits until no batch is in flight first. A micro-batch
 * whose solver call then needs more workspace fails with MAGMA_ERR_DEVICE_ALLOC,
 * and every request of that batch reports the code as its info. Returns
 * MAGMA_SUCCESS. */
magma_int_t magma_b200_server_set_workspace_limit(magma_b200_server_t server, size_t bytes);

/* Blocks until every submitted request has completed. */
magma_int_t magma_b200_server_drain(magma_b200_server_t server);

/* Counters: submitted, completed, micro-batches launched, peak device bytes in use. */
void magma_b200_server_stats(magma_b200_server_t server, long long* submitted, long long* completed,
                             long long* batches, long long* peak_bytes);

magma_int_t magma_b200_server_destroy(magma_b200_server_t server);

#ifdef __cplusplus
}
#endif

#endif /* MAGMA_B200_SERVE_H */
