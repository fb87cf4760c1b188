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

// Far-field testing of the batched complex64 apply on the tensor cores: per
// leaf box and tile of 32 RWGs, [Vf; (-khat) x Vf] (rows) times the box's Bm
// (J and M columns of every slot), contracted over the 3K pattern entries;
// adds c1 (L1J - K1M) + c2 (etai L2J - K2M) and c1 (K1J + L1M) + c2 (K2J +
// L2M / etai) into w (Code/MLFMM.cpp:285-351), whose near-field rows are
// already there.
struct LeafTcArg {
  const float2* Vf[2];           // receive patterns, complex64 [N][3K] (leaf order)
  const float2* Bm[2][kBatchSlots];  // leaf-level Bm of each slot, [B][6][K]
  const double* khat[2];         // [3][K]
  int K[2];
  const int* leaf_ptr;
  const int* leaf_rwg;
  double2* W;                    // w_j at W + j * ldw
  long long ldw;
  float2 c1, c2, etai;
  int N, R;
  int* status;
};

bool agg_tc_supported(const Plan& P, int R);
size_t agg_tc_smem_bytes(int kmax);
void launch_agg_tc(const Plan& P, const AggTcArg& a, cudaStream_t s);
void launch_leaf_tc(const Plan& P, const LeafTcArg& a, cudaStream_t s);

}  // namespace mlfma
