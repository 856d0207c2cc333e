// Magnus-integrator kernels (surf_magnus.f90:114-339), batched over angles.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace trhepd {

// m2 (V1 = V3 = nullptr) or m4 slice step from Vc (midpoint stage matrix) and its
// shared square S = Vc Vc: writes q (Qq), rp + r (+ m4 terms) (RPN), carries rp (RP).
void launch_magnus4_step(const cd* Vc, const cd* S, const cd* V1, const cd* V3, const cd* D,
                         int nang, int n, int ld, double h, double dz, double c0, double c1,
                         cd* Qq, cd* RPN, cd* RP, cudaStream_t st);
// m6 shared matrices of a slice: D13, S13 and the two exponent matrices Wm, Wp.
void launch_magnus6_shared(const cd* V1, const cd* V2, const cd* V3, int n, int ld, double d0,
                           double d1, cd* D13, cd* S13, cd* Wm, cd* Wp, cudaStream_t st);
// Per-angle (W + D_a)^2 from the shared S = W W.
void launch_magnus_square(const cd* S, const cd* W, const cd* D, int nang, int n, int ld, cd* R2,
                          cudaStream_t st);
// hyperbolic_exp6r of W + D_a from R2 = (W + D_a)^2 and T = R2 W.
void launch_magnus6_exp(const cd* W, const cd* D, const cd* R2, const cd* T, int nang, int n,
                        int ld, double h, const cd* RP, const cd* D13, const cd* M3s, double c0dz,
                        cd* Qq, cd* RPN, cd* RNEW, cudaStream_t st);
void launch_magnus6_carry(const cd* RNEW, const cd* D13, const cd* M3s, double c0dz, int nang,
                          int n, int ld, cd* RP, cudaStream_t st);
void launch_magnus6_m3(cd* M3s, const cd* S13, double cm, double c1dz, int n, int ld,
                       cudaStream_t st);
void launch_add(cd* A, const cd* B, int nang, int n, int ld, cudaStream_t st);

}  // namespace trhepd
