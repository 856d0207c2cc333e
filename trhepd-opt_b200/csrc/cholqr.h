// RK4 with CholeskyQR re-orthogonalisation (int_method 8, rk4_intgs,
// sim-trhepd-rheed/src/surf_rk.f90:93-156) on the angle-stacked state.
//
// The reference integrates [q; p] (column-major n x n blocks); the device keeps
// Q = q^H and P = p^H, row-major per angle, as for the other integrators.  In that
// layout the stage products are Q M with M = vvi2mate's matrix (vvi2matf's is its
// conjugate transpose), so the RK4 stages of int_method 7 serve unchanged.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace trhepd {

// invstrans (matcomp.f90:89-115) in the stacked layout: Q = (I + F^H) conj(G)^{-1},
// P = i (I - F^H), from F (nang x n x n, row-major).
void launch_invstrans_build(const cd* F, cd* Q, cd* P, const cd* gam, int nang, int n, int ld,
                            cudaStream_t st);
// strans (matcomp.f90:117-137) before matAdivB2: Q <- Q conj(G) - i P,
// P <- Q conj(G) + i P; the Gauss-Jordan solve that follows leaves P = f^H.
void launch_strans_build(cd* Q, cd* P, const cd* gam, int nang, int n, int ld, cudaStream_t st);

// power_est (matcomp.f90:530-594) per angle on [q; p]^H [q; p] = Q Q^H + P P^H with
// the vector x (nang x n) kept between calls.  steps < 0: x = (1 + i)/sqrt(2n) and
// every flag set (the CholeskyQR that follows the initial transform).  Else at most
// `steps` power steps, stopping as the reference does; dval[a] = the estimate,
// flag[a] = estimate > 1e2.
void launch_power_est(const cd* Q, const cd* P, cd* x, int* flag, double* dval, int nang, int n,
                      int ld, int steps, cudaStream_t st);

// bcgs / cqr (matgs.f90:5-35) for the flagged angles: G = Q Q^H + P P^H = L L^H
// (Cholesky, lower), then Q <- L^{-1} Q, P <- L^{-1} P (= (q R^{-1})^H, (p R^{-1})^H with
// R = L^H).  Scratch: cholqr_scratch_bytes(nang, n, ld).  A non-positive pivot of
// the Cholesky factor sets kStatusZeroPivot in *status.  Returns the launch count.
size_t cholqr_scratch_bytes(int nang, int n, int ld);
int launch_cholqr(cd* Q, cd* P, const int* flag, int nang, int n, int ld, void* scratch,
                  unsigned* status, cudaStream_t st);

}  // namespace trhepd
