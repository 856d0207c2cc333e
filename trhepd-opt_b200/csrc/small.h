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

// One problem of a fused launch: its RKN integration (hp_int_spa,
// surf_prkn.f90:278-330).  Q and P enter as the state after invstransh (Q = I)
// and leave as the state after the last half kick, as the stacked path leaves
// them.  The problem's CTAs are first_cta .. first_cta + nang - 1.
struct FusedProblem {
  cd* Q;
  cd* P;
  const TableEntry* table;  // ncol x nv stage table
  const int* pair;          // n x n beam-pair map (0-based table index)
  const cd* D;              // -conj(gamma^2) per angle (nang x ld)
  unsigned* status;
  int n, ld, nv, nang, ns;
  int interval;             // renormalisation interval of the growth-bound policy
  int first_cta;
  double dz;
};

// Problems of one fused launch, passed by value as a kernel parameter (CUDA
// 12 allows 32 KB of parameters): every angle of every problem, any mix of
// beam counts up to kFusedMaxBeams, one integrator (s stages, coefficients bab).
constexpr int kFusedMaxProblems = 192;
struct FusedLaunch {
  int nprob, s, policy, total_ctas;  // policy 0: Gershgorin test, 1: interval
  double bab[24];                    // Blanes-Moan coefficients b1, a1, b2, a2, ...
  FusedProblem p[kFusedMaxProblems];
};

// Launch the fused integration (one CTA per angle of every problem).  Returns
// the number of kernels launched.
int launch_fused_rkn(const FusedLaunch& L, cudaStream_t st);

}  // namespace trhepd
