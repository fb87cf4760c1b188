// Batched complex64 leaf aggregation on the tensor cores (agg_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include "plan.hpp"

namespace mlfma {

constexpr int kAggTcMaxRwgs = 64;  // RWGs per leaf box the shared-memory operands hold

struct AggTcArg {
  const float* Vs[2];            // radiation patterns, complex64 [N][3K] seen as real [N][6K]
  float2* S[2][kBatchSlots];     // leaf-level S of each slot, [B][6][K]
  int K[2];
  const int* leaf_ptr;
  const int* leaf_rwg;
  const double2* X;              // right-hand side j at X + j * ldx
  long long ldx;
  int N, R;
  int kmax;                      // RWGs per box rounded up to 8 (shared-memory sizing)
  int* status;
};

bool agg_tc_supported(const Plan& P, int R);
size_t agg_tc_smem_bytes(int kmax);
void launch_agg_tc(const Plan& P, const AggTcArg& a, cudaStream_t s);

}  // namespace mlfma
