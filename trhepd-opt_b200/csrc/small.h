// Fused small-beam surface integration: one CTA integrates one glancing angle
// through every slice with its state in shared memory (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace trhepd {

// Largest beam count of the fused kernel: Q, P and the stage matrix of one angle
// (64 x 64 complex each, padded rows) fill 202 KB of shared memory.
constexpr int kFusedMaxBeams = 64;

// One resident problem's RKN integration (hp_int_spa, surf_prkn.f90:278-330).
// Q and P enter as the state after invstransh (Q = I) and leave as the state
// after the last half kick, as the stacked path leaves them.
struct FusedRkn {
  cd* Q;
  cd* P;
  const TableEntry* table;  // ncol x nv stage table
  const int* pair;          // n x n beam-pair map (0-based table index)
  const cd* D;              // -conj(gamma^2) per angle (nang x ld)
  unsigned* status;
  int n, ld, nv, nang, ns, s;
  int policy;               // 0: Gershgorin test per slice, 1: every `interval` slices
  int interval;
  double dz;
  double bab[24];           // Blanes-Moan coefficients b1, a1, b2, a2, ...
};

// Launch the fused integration for every angle (one CTA each).  Returns the
// number of kernels launched.
int launch_fused_rkn(const FusedRkn& a, cudaStream_t st);

}  // namespace trhepd
