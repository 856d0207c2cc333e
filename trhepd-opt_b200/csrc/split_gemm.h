// Split-precision stage product on the tcgen05 tensor cores (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace trhepd {

struct SplitWorkspace {
  void* base = nullptr;
  int nang = 0, n = 0, slices = 0;
  unsigned* status = nullptr;  // device status word (kStatus* bits)
};

size_t split_workspace_bytes(int nang, int n, int slices);
// Carve the workspace and zero it on `st` (padded slice rows stay zero).
SplitWorkspace split_workspace_carve(void* base, int nang, int n, int slices, unsigned* status,
                                     cudaStream_t st);

// P += cb*(Q V + Q o D_a) with the potential product from BF16 slices; Qo = Q + ca*P.
// Returns the number of kernels launched.
int split_stage(const SplitWorkspace& w, const cd* Q, cd* P, cd* Qo, const cd* V, const cd* D,
                 int nang, int n, int ld, double cb, double ca, int slices, cudaStream_t st);

}  // namespace trhepd
