// Split-precision (INT8-sliced, tcgen05) chi0 contraction: host-side interface.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tg {

struct SplitArgs {
  const double2* A = nullptr;      // [np][ld] pair-block operands (FP64 complex)
  const double2* B = nullptr;
  int64_t ld = 0;
  int64_t np = 0;
  int n_pairs = 0;
  const int* pair_M = nullptr;     // host copies
  const int* pair_aoff = nullptr;
  const int64_t* pair_coff = nullptr;
  const int* d_pair_M = nullptr;   // device copies
  const int* d_pair_aoff = nullptr;
  const int64_t* d_pair_coff = nullptr;
  double2* C = nullptr;            // FP64 accumulator, C[pair_coff + u*M + v] += ...
  int num_sms = 148;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  int slices = 0;                  // 0 = default
};

size_t split_workspace_bytes(const SplitArgs& a);
cudaError_t launch_split_contraction(const SplitArgs& a, cudaStream_t s, int* launches);

}  // namespace tg
