// lu_tc.h -- host interface of the TMEM-resident tensor-core LU (lu_tc.cu).
#pragma once
#include "internal.h"

namespace mb200 {

struct TcLuArgs {
    int n, batch, lda;
    double** dA;       // FP64 inputs (read only)
    float* SA;         // FP32 U12 blocks (above the diagonal blocks), instance i at SA + i*n*n, ld n
    int** ipiv;        // pivots (1-based)
    int* sinfo;        // FP32 getrf info
    double* anrm;      // ||A||_inf
    int* iter;         // -2 on overflow of the conversion, else 0
    int* fail_count;   // instances for the FP64 fallback
    int* fail_list;
    int* err;          // set to 1 when a tensor-core wait timed out
    long long wait_limit;   // clock cycles a tensor-core completion wait may take
    int issue_mma;          // 0 only under the time-out test hook: no tensor-core work is issued
    // the refinement that follows each instance's factorisation in the same block
    int nrhs;
    double** dB;       // right-hand sides (read only)
    int ldb;
    double** dX;       // solutions
    int ldx;
};

bool lu_tc_supported(int n);
size_t lu_tc_smem_bytes();
magma_int_t lu_tc_launch(const TcLuArgs& args, cudaStream_t s);

}  // namespace mb200
