// tuning.h -- the kernel-variant table the dispatchers read, and its autotuner
// (tuning.cu). Takes the role of the reference's static tuning tables
// (control/batched_kernel_param.h, magmablas/gemm_config/*.h, tuned for one GPU)
// with a table measured on the device it runs on.
#pragma once
#include "internal.h"

namespace mb200 {

constexpr int kGemmBuckets = 4;   // max(M, N) <= 16, <= 32, <= 64, larger

constexpr int kLuBlockedBuckets = 4;   // blocked LU by max(m): <= 128, <= 256, <= 512, <= 1024
constexpr int kMixedTcOrders = 6;      // the tensor-core LU's orders: n = 96, 128, ..., 256

struct TuningTable {
    int gemm_variant[2][kGemmBuckets];   // [FP64, FP32][bucket]: tile variant (0: 64x64, 1: 32x32, 2: 16x16,
                                         // 3: the tensor cores, FP64 64x64 DMMA or FP32 128x128 tcgen05)
    int mixed_tc_lu;                     // 1: tensor-core LU in the mixed solve (where mixed_tc_n allows it)
    int lu_dmma[kLuBlockedBuckets];      // 1: FP64 blocked LU trailing update on the tensor cores (DMMA)
    int mixed_tc_n[kMixedTcOrders];      // per order n = 96 + 32 i: 1 tensor-core LU (+ fused refinement),
                                         // 0 CUDA-core FP32 LU + separate refinement
    int chol_queue;                      // variable-size FP64 Cholesky: 1 one persistent launch over all
                                         // sizes <= 512 (largest first), 0 one launch per size bucket
    int lu_queue;                        // variable-size FP64 getrf / gesv: the same choice
};

const TuningTable& tuning();   // defaults, or the file named by MAGMA_B200_TUNING, or the last autotune/set
TuningTable& tuning_mut();
constexpr int kTuningValuesV1 = 2 * kGemmBuckets + 1;
constexpr int kTuningValuesV2 = kTuningValuesV1 + kLuBlockedBuckets;
constexpr int kTuningValuesV3 = kTuningValuesV2 + kMixedTcOrders;
constexpr int kTuningValuesV4 = kTuningValuesV3 + 1;
constexpr int kTuningValues = kTuningValuesV4 + 1;

}  // namespace mb200
