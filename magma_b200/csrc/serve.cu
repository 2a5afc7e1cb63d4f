// serve.cu -- continuous-batching request loop for batched LU / Cholesky solves
// (include/magma_b200_serve.h). No counterpart in the reference.
//
// Requests are split into two size classes (n <= 128 and larger) so that small
// solves never wait behind the single-block factorisations of the largest ones;
// each class has its own FIFO, stream slots and completion thread. The parties
// share the server state under one mutex:
//   callers     submit requests into their class's FIFO (`pending`);
//   dispatcher  admits requests from the head of a FIFO while their device memory
//               (A, B, ipiv) fits in the arena (first-fit free list, shared by both
//               classes), takes everything admitted as one micro-batch, and launches
//               it on a free stream slot of that class: host->device copies, one
//               metadata upload, one variable-size LU call (magma_dgesv_vbatched_max_nocheck)
//               and one variable-size Cholesky call (magma_dposv_vbatched_max_nocheck),
//               result copies back, an event;
//   completers  (one per class) wait for their class's oldest in-flight batch, publish
//               its results, free their arena memory and the slot, and wake the dispatcher.
// With several slots per class, a batch's copies and kernels overlap the previous one's.
#include "internal.h"
#include "vbatched.h"
#include "../../include/magma_b200_serve.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace {

long long now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Identity matrices for the prewarm batch (instance i: n[i] x n[i], ld = n[i], at A + off[i]).
__global__ void prewarm_identity_kernel(double* A, const long long* off, const int* n, int count) {
    const int i = blockIdx.x;
    if (i >= count) return;
    const int ni = n[i];
    double* a = A + off[i];
    for (int idx = threadIdx.x; idx < ni * ni; idx += blockDim.x) a[idx] = (idx % (ni + 1) == 0) ? 1.0 : 0.0;
}

// Loads every kernel the request loop can launch before the first request: one LU and
// one Cholesky batch of identity matrices, one instance at each size-bucket edge, with
// 1 and with 4 right-hand sides (the two solve widths). Without it the first use of
// each kernel variant pays the driver's lazy module load inside some request's latency
// (measured: p99 20.6 ms instead of 0.63 ms for small requests). Best effort: skipped
// if its ~12 MB cannot be allocated.
void prewarm(magma_queue_t q, cudaStream_t s) {
    constexpr int kCount = 8;
    const int ns[kCount] = {8, 16, 32, 64, 128, 256, 512, 1024};
    std::vector<long long> offA(kCount), offB(kCount), offP(kCount);
    long long a = 0, b = 0, p = 0;
    for (int i = 0; i < kCount; ++i) {
        offA[i] = a; a += (long long)ns[i] * ns[i];
        offB[i] = b; b += (long long)ns[i] * 4;
        offP[i] = p; p += ns[i];
    }
    const size_t meta_ints = 4 * (kCount + 1) + kCount, bytes = 8 * (size_t)(a + b) + 4 * (size_t)p +
                                                                4 * meta_ints + 8 * 3 * kCount + 8 * kCount;
    char* d = nullptr;
    if (cudaMalloc(&d, bytes + 1024) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    double* dA = reinterpret_cast<double*>(d);
    double* dB = dA + a;
    int* dP = reinterpret_cast<int*>(dB + b);
    int* dN = dP + p;              // n[kCount+1]
    int* dR = dN + (kCount + 1);   // nrhs[kCount+1]
    int* dInfo = dR + (kCount + 1);
    long long* dOff = reinterpret_cast<long long*>(align256(reinterpret_cast<size_t>(dInfo + kCount + 1)));
    void** dPtr = reinterpret_cast<void**>(dOff + kCount);   // [A ptrs | B ptrs | ipiv ptrs]
    std::vector<void*> ptrs(3 * kCount);
    std::vector<int> hn(ns, ns + kCount);
    hn.push_back(0);
    for (int i = 0; i < kCount; ++i) {
        ptrs[i] = dA + offA[i];
        ptrs[kCount + i] = dB + offB[i];
        ptrs[2 * kCount + i] = dP + offP[i];
    }
    cudaMemcpyAsync(dN, hn.data(), sizeof(int) * (kCount + 1), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dOff, offA.data(), sizeof(long long) * kCount, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dPtr, ptrs.data(), sizeof(void*) * 3 * kCount, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(dB, 0, sizeof(double) * b, s);
    prewarm_identity_kernel<<<kCount, 256, 0, s>>>(dA, dOff, dN, kCount);
    double** pA = reinterpret_cast<double**>(dPtr);
    double** pB = pA + kCount;
    int** pP = reinterpret_cast<int**>(pA + 2 * kCount);
    for (int r : {1, 4}) {
        std::vector<int> hr(kCount, r);
        hr.push_back(0);
        cudaMemcpyAsync(dR, hr.data(), sizeof(int) * (kCount + 1), cudaMemcpyHostToDevice, s);
        magma_dgesv_vbatched_max_nocheck(dN, dR, pA, dN, pP, pB, dN, dInfo, kCount, 1024, r, q);
        magma_dposv_vbatched_max_nocheck(MagmaLower, dN, dR, pA, dN, pB, dN, dInfo, kCount, 1024, r, q);
        cudaStreamSynchronize(s);   // hr must outlive its copy
    }
    cudaFree(d);
    cudaGetLastError();
}

// First-fit allocator over [0, size) with coalescing of freed neighbours.
class Arena {
   public:
    explicit Arena(size_t size) { free_[0] = size; }
    bool alloc(size_t bytes, size_t* off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const size_t rest = it->second - bytes, start = it->first + bytes;
                free_.erase(it);
                if (rest) free_[start] = rest;
                used_ += bytes;
                peak_ = std::max(peak_, used_);
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t peak() const { return peak_; }

   private:
    std::map<size_t, size_t> free_;
    size_t used_ = 0, peak_ = 0;
};

struct Request {
    int kind, n, nrhs, lda, ldb, ldx;
    const double* A;
    const double* B;
    double* X;
    long long tag, t_submit = 0, t_done = 0;
    size_t off = 0, bytes = 0;
    int info = 0;
    size_t offA() const { return off; }
    size_t offB() const { return off + align256(sizeof(double) * n * n); }
    size_t offP() const { return offB() + align256(sizeof(double) * n * nrhs); }
    static size_t need(int n, int nrhs) {
        return align256(sizeof(double) * n * n) + align256(sizeof(double) * n * nrhs) + align256(sizeof(int) * n);
    }
};

// Per-batch metadata for one solver family (LU or Cholesky): size arrays with
// count+1 entries and pointer arrays, laid out back to back.
struct MetaLayout {
    size_t n, nrhs, lda, ldb, pa, pb, pp, info, bytes;
    explicit MetaLayout(int cap) {
        const size_t ints = align256(sizeof(int) * (cap + 1)), ptrs = align256(sizeof(void*) * cap);
        n = 0; nrhs = n + ints; lda = nrhs + ints; ldb = lda + ints;
        pa = ldb + ints; pb = pa + ptrs; pp = pb + ptrs; info = pp + ptrs; bytes = info + ints;
    }
};

struct Slot {
    cudaStream_t stream = nullptr;
    magma_queue_t queue = nullptr;
    cudaEvent_t done = nullptr;
    char* h_meta = nullptr;   // pinned: [LU meta][Cholesky meta]
    char* d_meta = nullptr;
    std::vector<Request*> reqs;
    bool busy = false;
    int cls = 0;              // size class this slot serves
    int rc[2] = {0, 0};       // return code of the batch's LU / Cholesky solver call
};

constexpr int kClasses = 2;
constexpr int kSmallN = 128;   // class 0: n <= kSmallN

}  // namespace

struct magma_b200_server {
    int device = 0, max_batch = 0;
    size_t budget = 0;
    char* arena_base = nullptr;
    Arena arena{0};
    std::vector<Slot> slots;
    MetaLayout meta{1};
    std::mutex mu;
    std::condition_variable cv_dispatch, cv_complete, cv_drain;
    std::deque<Request*> pending[kClasses];
    std::deque<Slot*> inflight[kClasses];
    int nclasses = 1;
    std::vector<Request*> finished;
    long long submitted = 0, completed = 0, batches = 0;
    bool stop = false;
    std::thread dispatcher, completer[kClasses];

    void dispatch_loop();
    void complete_loop(int cls);
    void launch(Slot& s);
};

void magma_b200_server::launch(Slot& s) {
    cudaSetDevice(device);
    // host -> device copies of every request's A and B (packed with ld = n)
    for (Request* r : s.reqs) {
        cudaMemcpy2DAsync(arena_base + r->offA(), sizeof(double) * r->n, r->A, sizeof(double) * r->lda,
                          sizeof(double) * r->n, r->n, cudaMemcpyHostToDevice, s.stream);
        cudaMemcpy2DAsync(arena_base + r->offB(), sizeof(double) * r->n, r->B, sizeof(double) * r->ldb,
                          sizeof(double) * r->n, r->nrhs, cudaMemcpyHostToDevice, s.stream);
    }
    // metadata for the two families
    int cnt[2] = {0, 0}, maxn[2] = {0, 0}, maxr[2] = {0, 0};
    for (int f = 0; f < 2; ++f) {
        char* h = s.h_meta + f * meta.bytes;
        int* n = reinterpret_cast<int*>(h + meta.n);
        int* nr = reinterpret_cast<int*>(h + meta.nrhs);
        int* la = reinterpret_cast<int*>(h + meta.lda);
        int* lb = reinterpret_cast<int*>(h + meta.ldb);
        void** pa = reinterpret_cast<void**>(h + meta.pa);
        void** pb = reinterpret_cast<void**>(h + meta.pb);
        void** pp = reinterpret_cast<void**>(h + meta.pp);
        for (Request* r : s.reqs) {
            if (r->kind != f) continue;
            const int i = cnt[f]++;
            n[i] = r->n; nr[i] = r->nrhs; la[i] = r->n; lb[i] = r->n;
            pa[i] = arena_base + r->offA();
            pb[i] = arena_base + r->offB();
            pp[i] = arena_base + r->offP();
            maxn[f] = std::max(maxn[f], r->n);
            maxr[f] = std::max(maxr[f], r->nrhs);
        }
    }
    cudaMemcpyAsync(s.d_meta, s.h_meta, 2 * meta.bytes, cudaMemcpyHostToDevice, s.stream);
    s.rc[0] = s.rc[1] = 0;
    for (int f = 0; f < 2; ++f) {
        if (!cnt[f]) continue;
        char* d = s.d_meta + f * meta.bytes;
        auto I = [&](size_t o) { return reinterpret_cast<int*>(d + o); };
        auto P = [&](size_t o) { return reinterpret_cast<double**>(d + o); };
        if (f == MAGMA_B200_SOLVE_LU)
            s.rc[f] = magma_dgesv_vbatched_max_nocheck(I(meta.n), I(meta.nrhs), P(meta.pa), I(meta.lda),
                                             reinterpret_cast<int**>(d + meta.pp), P(meta.pb), I(meta.ldb),
                                             I(meta.info), cnt[f], maxn[f], maxr[f], s.queue);
        else
            s.rc[f] = magma_dposv_vbatched_max_nocheck(MagmaLower, I(meta.n), I(meta.nrhs), P(meta.pa), I(meta.lda),
                                             P(meta.pb), I(meta.ldb), I(meta.info), cnt[f], maxn[f], maxr[f],
                                             s.queue);
    }
    // results back: X and info
    for (Request* r : s.reqs)
        cudaMemcpy2DAsync(r->X, sizeof(double) * r->ldx, arena_base + r->offB(), sizeof(double) * r->n,
                          sizeof(double) * r->n, r->nrhs, cudaMemcpyDeviceToHost, s.stream);
    for (int f = 0; f < 2; ++f)
        if (cnt[f])
            cudaMemcpyAsync(s.h_meta + f * meta.bytes + meta.info, s.d_meta + f * meta.bytes + meta.info,
                            sizeof(int) * cnt[f], cudaMemcpyDeviceToHost, s.stream);
    cudaEventRecord(s.done, s.stream);
}

void magma_b200_server::dispatch_loop() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        Slot* free_slot = nullptr;
        int cls = 0;
        cv_dispatch.wait(lk, [&] {
            if (stop) return true;
            // the class whose head request is oldest among those that can go now
            long long best = 0;
            free_slot = nullptr;
            for (int c = 0; c < nclasses; ++c) {
                if (pending[c].empty()) continue;
                Slot* fs = nullptr;
                for (Slot& sl : slots)
                    if (!sl.busy && sl.cls == c) { fs = &sl; break; }
                if (!fs) continue;
                size_t off;   // can the head be admitted now?
                if (!arena.alloc(pending[c].front()->bytes, &off)) continue;
                arena.release(off, pending[c].front()->bytes);
                if (!free_slot || pending[c].front()->t_submit < best) {
                    free_slot = fs;
                    cls = c;
                    best = pending[c].front()->t_submit;
                }
            }
            return free_slot != nullptr;
        });
        if (stop) return;
        Slot& s = *free_slot;
        s.reqs.clear();
        std::deque<Request*>& q = pending[cls];
        while (!q.empty() && (int)s.reqs.size() < max_batch) {
            Request* r = q.front();
            if (!arena.alloc(r->bytes, &r->off)) break;   // FIFO admission by memory budget
            q.pop_front();
            s.reqs.push_back(r);
        }
        s.busy = true;
        ++batches;
        lk.unlock();
        launch(s);
        lk.lock();
        inflight[cls].push_back(&s);
        cv_complete.notify_all();
    }
}

void magma_b200_server::complete_loop(int cls) {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv_complete.wait(lk, [&] { return stop || !inflight[cls].empty(); });
        if (inflight[cls].empty() && stop) return;
        Slot* s = inflight[cls].front();
        lk.unlock();
        cudaEventSynchronize(s->done);
        const long long t = now_ns();
        lk.lock();
        inflight[cls].pop_front();
        int idx[2] = {0, 0};
        for (Request* r : s->reqs) {
            const int* info = reinterpret_cast<const int*>(s->h_meta + r->kind * meta.bytes + meta.info);
            const int k = idx[r->kind]++;
            // a failed solver call leaves no info behind: report its MAGMA error code instead
            r->info = s->rc[r->kind] != 0 ? s->rc[r->kind] : info[k];
            r->t_done = t;
            arena.release(r->off, r->bytes);
            finished.push_back(r);
            ++completed;
        }
        s->reqs.clear();
        s->busy = false;
        cv_dispatch.notify_all();
        cv_drain.notify_all();
    }
}

extern "C" {

magma_int_t magma_b200_server_create(magma_int_t device, size_t budget_bytes, magma_int_t streams,
                                     magma_int_t max_batch, magma_b200_server_t* out) {
    if (streams < 1 || max_batch < 1 || budget_bytes < 4096) return MAGMA_ERR_ILLEGAL_VALUE;
    cudaSetDevice(device);
    auto* sv = new magma_b200_server();
    sv->device = device;
    sv->max_batch = max_batch;
    sv->meta = MetaLayout(max_batch);
    if (cudaMalloc(&sv->arena_base, budget_bytes) != cudaSuccess) {
        cudaGetLastError();
        delete sv;
        return MAGMA_ERR_DEVICE_ALLOC;
    }
    sv->arena = Arena(budget_bytes);
    sv->budget = budget_bytes;
    sv->slots.resize(streams);
    for (Slot& s : sv->slots) {
        cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
        magma_queue_create_from_cuda_internal(device, s.stream, nullptr, nullptr, &s.queue, "server", __FILE__,
                                              __LINE__);
        // bucket lists of the vbatched calls: reserve once so batches never grow the workspace
        magma_queue_reserve_workspace(s.queue, sizeof(int) * (mb200::bucketize_ws_ints(max_batch, 16) +
                                                              mb200::bucket_sort_ws_ints(max_batch, 16)));
        cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
        if (cudaHostAlloc(reinterpret_cast<void**>(&s.h_meta), 2 * sv->meta.bytes, cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaMalloc(&s.d_meta, 2 * sv->meta.bytes) != cudaSuccess) {
            cudaGetLastError();
            magma_b200_server_destroy(sv);
            return MAGMA_ERR_DEVICE_ALLOC;
        }
    }
    prewarm(sv->slots[0].queue, sv->slots[0].stream);
    // two size classes when there are at least two stream slots (slots alternate classes)
    sv->nclasses = streams >= 2 ? kClasses : 1;
    for (int i = 0; i < (int)sv->slots.size(); ++i) sv->slots[i].cls = i % sv->nclasses;
    sv->dispatcher = std::thread([sv] { sv->dispatch_loop(); });
    for (int c = 0; c < sv->nclasses; ++c) sv->completer[c] = std::thread([sv, c] { sv->complete_loop(c); });
    *out = sv;
    return MAGMA_SUCCESS;
}

magma_int_t magma_b200_server_submit(magma_b200_server_t sv, magma_int_t kind, magma_int_t n, magma_int_t nrhs,
                                     const double* A, magma_int_t lda, const double* B, magma_int_t ldb, double* X,
                                     magma_int_t ldx, long long tag) {
    if (kind != MAGMA_B200_SOLVE_LU && kind != MAGMA_B200_SOLVE_CHOLESKY) return -1;
    if (n < 1) return -2;
    if (nrhs < 1) return -3;
    if (!A) return -4;
    if (lda < n) return -5;
    if (!B) return -6;
    if (ldb < n) return -7;
    if (!X) return -8;
    if (ldx < n) return -9;
    if (n > 1024) return MAGMA_ERR_NOT_SUPPORTED;
    auto* r = new Request{(int)kind, (int)n, (int)nrhs, (int)lda, (int)ldb, (int)ldx, A, B, X, tag};
    r->bytes = Request::need(n, nrhs);
    if (r->bytes > sv->budget) {   // could never be admitted
        delete r;
        return MAGMA_ERR_NOT_SUPPORTED;
    }
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        r->t_submit = now_ns();
        sv->pending[(sv->nclasses > 1 && n > kSmallN) ? 1 : 0].push_back(r);
        ++sv->submitted;
    }
    sv->cv_dispatch.notify_one();
    return MAGMA_SUCCESS;
}

magma_int_t magma_b200_server_poll(magma_b200_server_t sv, long long* tags, magma_int_t* infos, long long* t_submit,
                                   long long* t_done, magma_int_t max) {
    std::lock_guard<std::mutex> lk(sv->mu);
    const int k = std::min<int>(max, (int)sv->finished.size());
    for (int i = 0; i < k; ++i) {
        Request* r = sv->finished[i];
        tags[i] = r->tag;
        infos[i] = r->info;
        t_submit[i] = r->t_submit;
        t_done[i] = r->t_done;
        delete r;
    }
    sv->finished.erase(sv->finished.begin(), sv->finished.begin() + k);
    return k;
}

magma_int_t magma_b200_server_drain(magma_b200_server_t sv) {
    std::unique_lock<std::mutex> lk(sv->mu);
    sv->cv_drain.wait(lk, [&] { return sv->completed == sv->submitted; });
    return MAGMA_SUCCESS;
}

magma_int_t magma_b200_server_set_workspace_limit(magma_b200_server_t sv, size_t bytes) {
    std::unique_lock<std::mutex> lk(sv->mu);
    // no batch in flight: the dispatcher marks a slot busy under this lock before launching
    sv->cv_drain.wait(lk, [&] {
        for (const Slot& s : sv->slots)
            if (s.busy) return false;
        return true;
    });
    cudaSetDevice(sv->device);
    for (Slot& s : sv->slots) magma_b200_queue_set_workspace_limit(s.queue, bytes);
    return MAGMA_SUCCESS;
}

void magma_b200_server_stats(magma_b200_server_t sv, long long* submitted, long long* completed, long long* batches,
                             long long* peak_bytes) {
    std::lock_guard<std::mutex> lk(sv->mu);
    *submitted = sv->submitted;
    *completed = sv->completed;
    *batches = sv->batches;
    *peak_bytes = (long long)sv->arena.peak();
}

magma_int_t magma_b200_server_destroy(magma_b200_server_t sv) {
    if (!sv) return MAGMA_SUCCESS;
    if (sv->dispatcher.joinable()) magma_b200_server_drain(sv);
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_dispatch.notify_all();
    sv->cv_complete.notify_all();
    if (sv->dispatcher.joinable()) sv->dispatcher.join();
    for (auto& c : sv->completer)
        if (c.joinable()) c.join();
    for (Slot& s : sv->slots) {
        if (s.queue) magma_queue_destroy_internal(s.queue, "server", __FILE__, __LINE__);
        if (s.stream) cudaStreamDestroy(s.stream);
        if (s.done) cudaEventDestroy(s.done);
        if (s.h_meta) cudaFreeHost(s.h_meta);
        if (s.d_meta) cudaFree(s.d_meta);
    }
    for (Request* r : sv->finished) delete r;
    if (sv->arena_base) cudaFree(sv->arena_base);
    delete sv;
    return MAGMA_SUCCESS;
}

}  // extern "C"
