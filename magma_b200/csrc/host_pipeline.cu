// host_pipeline.cu -- batched solves of systems that live in host memory, with the
// transfers pipelined against the solves (magma_b200_host_solver_*).
//
// No reference counterpart: MAGMA's batched routines take device pointer arrays
// only, and its testers upload, solve and read back in sequence
// (testing/testing_zgesv_batched.cpp:111-125). Here the batch is cut into chunks.
// Every chunk's upload is queued on one copy stream, back to back, so the
// host-to-device link never idles; chunk c is solved on the queue's stream as soon
// as its upload has landed (an event), and its results go back on a second copy
// stream while later chunks are still uploading or solving. Each solver kernel
// works instance by instance, so the results equal one call over the whole batch.
// The staging buffers, pointer arrays, streams and events are created once per
// solver. A solve returns once everything is queued; the queue's stream waits for
// the last read-back, so synchronising the queue covers the whole sequence. Host
// buffers should be page-locked (cudaHostAlloc / cudaHostRegister): pageable memory
// gives the same results, but the copies then stage through the driver and do
// not overlap the solves.
#include "internal.h"
#include "../../include/magma_b200.h"
#include <vector>

struct magma_b200_host_solver {
    int kind = 0, batch = 0, n = 0, nrhs = 0, lda = 0, ldb = 0;
    magma_queue_t queue = nullptr;
    double *A = nullptr, *B = nullptr, *X = nullptr;
    int *ipiv = nullptr, *iter = nullptr, *info = nullptr;
    void** ptrs = nullptr;   // [A | B | X | ipiv] pointer arrays, batch each
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t start = nullptr;
    std::vector<cudaEvent_t> landed, solved;
    std::vector<int> c0;     // chunk starts, then batch
};

namespace {

template <typename T>
bool dev_alloc(T** p, size_t count) {
    if (cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (count ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return false;
    }
    return true;
}

void release(magma_b200_host_solver* s) {
    if (!s) return;
    if (s->up) cudaStreamSynchronize(s->up);
    if (s->down) cudaStreamSynchronize(s->down);
    for (void* p : {(void*)s->A, (void*)s->B, (void*)s->X, (void*)s->ipiv, (void*)s->iter, (void*)s->info,
                    (void*)s->ptrs})
        if (p) cudaFree(p);
    for (cudaEvent_t e : s->landed) cudaEventDestroy(e);
    for (cudaEvent_t e : s->solved) cudaEventDestroy(e);
    if (s->start) cudaEventDestroy(s->start);
    if (s->up) cudaStreamDestroy(s->up);
    if (s->down) cudaStreamDestroy(s->down);
    delete s;
}

}  // namespace

extern "C" {

magma_int_t magma_b200_host_solver_create(magma_int_t kind, magma_int_t batch, magma_int_t n, magma_int_t nrhs,
                                          magma_int_t lda, magma_int_t ldb, magma_int_t chunks, magma_queue_t queue,
                                          magma_b200_host_solver_t* solver) {
    if (kind != MAGMA_B200_HOST_DSGESV && kind != MAGMA_B200_HOST_DGESV) return -1;
    if (batch < 1) return -2;
    if (n < 1) return -3;
    if (nrhs < 1) return -4;
    if (lda < n) return -5;
    if (ldb < n) return -6;
    if (chunks < 1) return -7;
    if (!queue) return -8;
    if (!solver) return -9;
    auto* s = new magma_b200_host_solver();
    s->kind = kind; s->batch = batch; s->n = n; s->nrhs = nrhs; s->lda = lda; s->ldb = ldb; s->queue = queue;
    cudaSetDevice(queue->device);
    const size_t sa = (size_t)n * lda, sb = (size_t)nrhs * ldb, sx = (size_t)nrhs * n;
    bool ok = dev_alloc(&s->A, sa * batch) && dev_alloc(&s->B, sb * batch) && dev_alloc(&s->ipiv, (size_t)n * batch) &&
              dev_alloc(&s->info, batch) && dev_alloc(&s->ptrs, 4 * (size_t)batch);
    if (ok && kind == MAGMA_B200_HOST_DSGESV) ok = dev_alloc(&s->X, sx * batch) && dev_alloc(&s->iter, batch);
    if (!ok) {
        release(s);
        return MAGMA_ERR_DEVICE_ALLOC;
    }
    std::vector<void*> p(4 * (size_t)batch, nullptr);
    for (int i = 0; i < batch; ++i) {
        p[i] = s->A + i * sa;
        p[batch + i] = s->B + i * sb;
        p[2 * batch + i] = s->X ? static_cast<void*>(s->X + i * sx) : nullptr;
        p[3 * batch + i] = s->ipiv + (size_t)i * n;
    }
    ok = cudaMemcpy(s->ptrs, p.data(), sizeof(void*) * p.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking) == cudaSuccess &&
         cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&s->start, cudaEventDisableTiming) == cudaSuccess;
    const int per = (batch + chunks - 1) / chunks;
    for (int c0 = 0; ok && c0 < batch; c0 += per) {
        s->c0.push_back(c0);
        cudaEvent_t a = nullptr, b = nullptr;
        ok = cudaEventCreateWithFlags(&a, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&b, cudaEventDisableTiming) == cudaSuccess;
        if (a) s->landed.push_back(a);
        if (b) s->solved.push_back(b);
    }
    s->c0.push_back(batch);
    if (!ok) {
        cudaGetLastError();
        release(s);
        return MAGMA_ERR_UNKNOWN;
    }
    *solver = s;
    return MAGMA_SUCCESS;
}

magma_int_t magma_b200_host_solve(magma_b200_host_solver_t s, const double* hA, const double* hB, double* hX,
                                  magma_int_t* hI, magma_int_t* hInfo) {
    if (!s) return -1;
    if (!hA) return -2;
    if (!hB) return -3;
    if (!hX) return -4;
    if (!hI) return -5;
    if (!hInfo) return -6;
    cudaSetDevice(s->queue->device);
    const cudaStream_t q = s->queue->stream;
    const size_t sa = (size_t)s->n * s->lda, sb = (size_t)s->nrhs * s->ldb, sx = (size_t)s->nrhs * s->n;
    const bool mixed = s->kind == MAGMA_B200_HOST_DSGESV;
    double** pA = reinterpret_cast<double**>(s->ptrs);
    double** pB = pA + s->batch;
    double** pX = pB + s->batch;
    int** pP = reinterpret_cast<int**>(pX + s->batch);
    const int chunks = (int)s->c0.size() - 1;
    cudaEventRecord(s->start, q);              // earlier work on the staging buffers comes first
    cudaStreamWaitEvent(s->up, s->start, 0);
    cudaStreamWaitEvent(s->down, s->start, 0);
    for (int c = 0; c < chunks; ++c) {         // every upload, back to back
        const size_t i0 = s->c0[c], cnt = s->c0[c + 1] - s->c0[c];
        cudaMemcpyAsync(s->A + i0 * sa, hA + i0 * sa, sizeof(double) * sa * cnt, cudaMemcpyHostToDevice, s->up);
        cudaMemcpyAsync(s->B + i0 * sb, hB + i0 * sb, sizeof(double) * sb * cnt, cudaMemcpyHostToDevice, s->up);
        cudaEventRecord(s->landed[c], s->up);
    }
    magma_int_t rc = MAGMA_SUCCESS;
    for (int c = 0; c < chunks; ++c) {         // each chunk solved once it has landed, then read back
        const int i0 = s->c0[c], cnt = s->c0[c + 1] - s->c0[c];
        cudaStreamWaitEvent(q, s->landed[c], 0);
        const magma_int_t r =
            mixed ? magma_dsgesv_batched(s->n, s->nrhs, pA + i0, s->lda, pP + i0, pB + i0, s->ldb, pX + i0, s->n,
                                         s->iter + i0, s->info + i0, cnt, s->queue)
                  : magma_dgesv_batched(s->n, s->nrhs, pA + i0, s->lda, pP + i0, pB + i0, s->ldb, s->info + i0, cnt,
                                        s->queue);
        if (r != MAGMA_SUCCESS && rc == MAGMA_SUCCESS) rc = r;   // the first error
        cudaEventRecord(s->solved[c], q);
        cudaStreamWaitEvent(s->down, s->solved[c], 0);
        if (mixed) {
            cudaMemcpyAsync(hX + i0 * sx, s->X + i0 * sx, sizeof(double) * sx * cnt, cudaMemcpyDeviceToHost, s->down);
            cudaMemcpyAsync(hI + i0, s->iter + i0, sizeof(int) * cnt, cudaMemcpyDeviceToHost, s->down);
        } else {
            cudaMemcpyAsync(hX + i0 * sb, s->B + i0 * sb, sizeof(double) * sb * cnt, cudaMemcpyDeviceToHost, s->down);
            cudaMemcpyAsync(hI + (size_t)i0 * s->n, s->ipiv + (size_t)i0 * s->n, sizeof(int) * s->n * cnt,
                            cudaMemcpyDeviceToHost, s->down);
        }
        cudaMemcpyAsync(hInfo + i0, s->info + i0, sizeof(int) * cnt, cudaMemcpyDeviceToHost, s->down);
    }
    cudaEventRecord(s->start, s->down);        // the queue's stream covers the read-backs
    cudaStreamWaitEvent(q, s->start, 0);
    if (rc == MAGMA_SUCCESS) rc = mb200::launch_status();
    return rc;
}

magma_int_t magma_b200_host_solver_chunk_start(magma_b200_host_solver_t s, magma_int_t c) {
    if (!s || c < 0 || c >= (magma_int_t)s->c0.size()) return -1;
    return s->c0[c];
}

magma_int_t magma_b200_host_solver_destroy(magma_b200_host_solver_t s) {
    if (!s) return -1;
    release(s);
    return MAGMA_SUCCESS;
}

}  // extern "C"
