// vbatched.h -- device-side size checks, reductions and bucketing shared by
// the variable-size entry points.
#pragma once
#include "internal.h"
#include <climits>

namespace mb200 {

struct BucketEdges {
    static constexpr int kMax = 16;
    int n;
    int e[kMax];
};

// Counting-sorts instances 0..batch-1 into nb buckets by key[i] (bucket b
// holds keys <= edges[b]; keys <= 0 are dropped). ws must hold
// bucketize_ws_ints(batch, nb) ints. Outputs device pointers to the counts
// (nb ints, followed by nb more ints set to zero that callers may use as
// counters) and the lists (bucket b at lists + b*batch).
magma_int_t bucketize(const int* key, int batch, const int* edges_host, int nb, cudaStream_t s, int* ws,
                      int** counts_out, int** lists_out);
size_t bucketize_ws_ints(int batch, int nb);
// As bucketize, keyed by max(key[i], key2[i]) (instances with a key <= 0 in either are dropped).
magma_int_t bucketize2(const int* key, const int* key2, int batch, const int* edges_host, int nb, cudaStream_t s,
                       int* ws, int** counts_out, int** lists_out);

// Reorders every bucket's list (as bucketize / bucketize2 left it) by key descending,
// so that the kernels' blocks, walking a list round-robin, start on the costliest
// instances and finish together (largest-first). tmp must hold
// bucket_sort_ws_ints(batch, nb) ints. Keys above a bucket's lower edge + 1023 share
// the first place. The instances themselves are unchanged: each is processed alone.
magma_int_t sort_buckets_desc(const int* key, const int* key2, int batch, const int* edges_host, int nb,
                              cudaStream_t s, const int* counts, int* lists, int* tmp);
size_t bucket_sort_ws_ints(int batch, int nb);

// out[0..2] = max of a, b, c (null arrays give 0), out[3..5] = their minima. Synchronises the queue.
magma_int_t reduce_sizes(const int* a, const int* b, const int* c, int batch, magma_queue_t queue, int out[6]);
// *out = min over i of ld[i] - rows[i]. Synchronises the queue.
magma_int_t ld_slack(const int* rows, const int* ld, int batch, magma_queue_t queue, int* out);
// as ld_slack with max(1, rows[i]) in place of rows[i] (the checks written ld < max(1, rows))
magma_int_t ld_slack1(const int* rows, const int* ld, int batch, magma_queue_t queue, int* out);

// Blocks of `kernel` that fit on the whole GPU at once.
int resident_blocks(const void* kernel, int threads, size_t smem);

}  // namespace mb200
