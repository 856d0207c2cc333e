// Bulk reflection matrices (blkref, sim-trhepd-rheed/src/bulk.f90:7-128) on the GPU.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.h"

namespace trhepd {

// C_b = alpha A_b B_b + beta C_b, row-major complex, for b < batch (items with
// active[b] == 0 skipped when active is given).  beta must be 0 or 1.
struct BatchedGemm {
  const cd* A;
  const cd* B;
  cd* C;
  int M, N, K, lda, ldb, ldc;
  long long sA, sB, sC;  // element strides between batch items
  cd alpha;
  int beta;
  int batch;
  const int* active;
};
void launch_zgemm_batched(const BatchedGemm& g, cudaStream_t st);

// items b = angle * ngr + group, every matrix padded to n x n (ld) / 2n x 2n (ld2)
void launch_bulk_hamiltonian(const TableEntry* tcol, const int* pair, const cd* gam,
                             const int* gsize, int ngr, int n, int ld, int batch, double h2, cd* H,
                             cd* X, cudaStream_t st);
void launch_bulk_poly(const cd* X, const cd* X2, const cd* X3, const cd* X4, const double* c,
                      int n, int ld, int batch, cd* out, cudaStream_t st);
void launch_bulk_axpby(cd* A, const cd* B, double alpha, double beta, double diag, int n, int ld,
                       int batch, cudaStream_t st);
void launch_bulk_build_e(const cd* C, const cd* S, const cd* Hs, int n, int ld, int ld2, int batch,
                         cd* E, cudaStream_t st);
void launch_bulk_similarity(const cd* E, const cd* gam, const cd* phase, const int* gsize, int ngr,
                            int n, int ld2, int batch, cd* T, cudaStream_t st);
void launch_bulk_phase_cols(cd* T, const cd* phase, const int* gsize, int ngr, int n, int ld2,
                            int batch, cudaStream_t st);
void launch_bulk_layer_init(const cd* T, const int* active, int n, int ld, int ld2, int batch,
                            cd* t1, cd* t2, cudaStream_t st);
void launch_bulk_transpose_pair(const cd* t1, const cd* t2, const int* active, const int* gsize,
                                int ngr, int n, int ld, int batch, cd* Q, cd* P, cudaStream_t st);
void launch_bulk_layer_finish(const cd* P, int* active, const int* gsize, int ngr, int n, int ld,
                              int batch, int layer, double epsb, double* r20, cd* R,
                              cudaStream_t st);

}  // namespace trhepd
