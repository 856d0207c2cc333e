// Split-precision stage product on the tcgen05 tensor cores (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace trhepd {

struct SplitWorkspace {
  void* base = nullptr;
  int nang = 0, n = 0, slices = 0;
  unsigned* status = nullptr;  // device status word (kStatus* bits)
  int max_ctas = 0;            // persistent kernels: at most this many CTAs (0: one per SM)
};

size_t split_workspace_bytes(int nang, int n, int slices, int nprob = 1);
// Carve the workspace and zero it on `st` (padded slice rows stay zero).
SplitWorkspace split_workspace_carve(void* base, int nang, int n, int slices, unsigned* status,
                                     cudaStream_t st, int nprob = 1);

// Tensor-core kernel forms of the stage product.
//   kSplitPersistent: one CTA per SM over all tiles; the accumulators of a tile
//     are drained to registers and the FP64 update runs during the next tile's MMAs;
//   kSplitPerTile: one CTA per tile, the epilogue after the tile's MMAs.
// Both use three FP32 accumulators (slice pairs with s+t = 0, 1, >= 2).
//   kSplitInt8: the persistent form on signed 8-bit digits (kind::i8), one exact
//     INT32 accumulator per digit level s+t (3 or 4 slices).
enum SplitVariant { kSplitPersistent = 0, kSplitPerTile = 1, kSplitInt8 = 2 };

// P += cb*(Q V + Q o D_a) with the potential product from BF16 or INT8 slices;
// Qo = Q + ca*P.  When `ev` is given, ev[0] and ev[1] are recorded around the
// tensor-core kernel.  Returns the number of kernels launched.
int split_stage(const SplitWorkspace& w, const cd* Q, cd* P, cd* Qo, const cd* V, const cd* D,
                int nang, int n, int ld, double cb, double ca, int slices, int variant,
                const cudaEvent_t* ev, cudaStream_t st, StackedRows sr = {});

}  // namespace trhepd
