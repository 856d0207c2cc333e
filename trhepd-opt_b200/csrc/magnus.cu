// Elementwise kernels of the Magnus integrators (surf_magnus.f90:114-339) on
// the GPU, batched over angles.
//
// Per angle a the stage matrix is M_a = V + diag(D_a): V (n x ld, shared by every
// angle, from the K4 gather) and D_a = -conj(gamma^2) (Pb.D).  The matrix
// functions of M_a that hyperbolic_exp4r/6r (matcomp.f90:388-428) need are
// formed from one shared product per slice,
//     (W + D_a)^2 = W^2 + D_a W + W D_a + D_a^2      (W^2 shared),
//     (W + D_a)^3 = (W + D_a)^2 W + (W + D_a)^2 D_a  (one batched product),
// so only the state updates P += Q rp, Q += P q and the cube are per-angle
// GEMMs (batched FP64 DMMA, bulk.cu).  Matrices are row-major: per angle
// [nang][n][ld], shared [n][ld].
#include <cuda_runtime.h>

#include "magnus.h"

namespace trhepd {

namespace {

__device__ __forceinline__ cd mval(const cd* V, const cd* D, int a, int i, int j, int ld) {
  cd m = V[(size_t)i * ld + j];
  if (i == j) m = m + D[(size_t)a * ld + j];
  return m;
}

// (W + D_a)^2 from the shared W^2 (element (i, j) of angle a).
__device__ __forceinline__ cd square_elem(const cd* S, const cd* W, const cd* D, int a, int i,
                                          int j, int ld) {
  const cd di = D[(size_t)a * ld + i], dj = D[(size_t)a * ld + j];
  const cd w = W[(size_t)i * ld + j];
  cd r = S[(size_t)i * ld + j] + di * w + w * dj;
  if (i == j) r = r + di * di;
  return r;
}

// m2 / m4 slice step: hyperbolic_exp4r(h, M) with M = Vc + D_a,
//   q = h^3/6 M + h^5/120 M^2 + h I,   r = h/2 M - h^3/24 M^2,
// then rpn = rp + r + e1 (the vector added before P += Q rpn) and
// rp <- r + e2 (carried to the next slice), with e1, e2 from the m4 Gauss-point
// differences (zero for m2).
__global__ void k_magnus4_step(const cd* __restrict__ Vc, const cd* __restrict__ S,
                               const cd* __restrict__ V1, const cd* __restrict__ V3,
                               const cd* __restrict__ D, int n, int ld, double h, double dz,
                               double c0, double c1, cd* __restrict__ Qq, cd* __restrict__ RPN,
                               cd* __restrict__ RP) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (j >= n) return;
  const int a = r / n, i = r - a * n;
  const size_t o = (size_t)r * ld + j;
  const cd m = mval(Vc, D, a, i, j, ld);
  const cd m2 = square_elem(S, Vc, D, a, i, j, ld);
  const double h3 = h * h * h, h5 = h3 * h * h;
  cd q = (h3 / 6) * m + (h5 / 120) * m2;
  if (i == j) q = q + cd{h, 0.0};
  const cd rr = (h / 2) * m - (h3 / 24) * m2;
  cd rpn, rpx;
  if (V1) {  // m4: m1 <- m3 - m1, m3 <- m1 - 2 m2 + m3 (surf_magnus.f90:194-199)
    const cd g1 = mval(V1, D, a, i, j, ld), g3 = mval(V3, D, a, i, j, ld);
    const cd d13 = g3 - g1;
    const cd s13 = g1 - 2.0 * m + g3;
    rpn = RP[o] + rr + dz * (-c0 * d13 + c1 * s13);
    rpx = rr + dz * (c0 * d13 + c1 * s13);
  } else {  // m2
    rpn = RP[o] + rr;
    rpx = rr;
  }
  Qq[o] = q;
  RPN[o] = rpn;
  RP[o] = rpx;
}

// m6 shared matrices of a slice (surf_magnus.f90:267-276):
//   D13 = V3 - V1, S13 = V1 - 2 V2 + V3, W2 = V2 + d1 S13,
//   Wm = W2 - d0 D13, Wp = W2 + d0 D13 (the matrices whose exponentials are taken).
__global__ void k_magnus6_shared(const cd* __restrict__ V1, const cd* __restrict__ V2,
                                 const cd* __restrict__ V3, int n, int ld, double d0, double d1,
                                 cd* __restrict__ D13, cd* __restrict__ S13, cd* __restrict__ Wm,
                                 cd* __restrict__ Wp) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (j >= n) return;
  const size_t o = (size_t)i * ld + j;
  const cd d13 = V3[o] - V1[o];
  const cd s13 = V1[o] - 2.0 * V2[o] + V3[o];
  const cd w2 = V2[o] + d1 * s13;
  D13[o] = d13;
  S13[o] = s13;
  Wm[o] = w2 - d0 * d13;
  Wp[o] = w2 + d0 * d13;
}

// Per-angle square (W + D_a)^2 into R2.
__global__ void k_magnus_square(const cd* __restrict__ S, const cd* __restrict__ W,
                                const cd* __restrict__ D, int n, int ld, cd* __restrict__ R2) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (j >= n) return;
  const int a = r / n, i = r - a * n;
  R2[(size_t)r * ld + j] = square_elem(S, W, D, a, i, j, ld);
}

// hyperbolic_exp6r(h, W + D_a) given R2 = (W + D_a)^2 and T = R2 W (the D_a part
// of the cube is added here):
//   q = h^3 cq0 M + h^5 cq1 M^2 + h^7 cq2 M^3 + h I,  r = h cr0 M + h^3 cr1 M^2 + h^5 cr2 M^3,
// then rp <- rp + r + add (add = -c0 dz D13 + M3s for the first half step, 0 for
// the second), writing RPN; RNEW <- r.
__global__ void k_magnus6_exp(const cd* __restrict__ W, const cd* __restrict__ D,
                              const cd* __restrict__ R2, const cd* __restrict__ T, int n, int ld,
                              double h, const cd* __restrict__ RP, const cd* __restrict__ D13,
                              const cd* __restrict__ M3s, double c0dz, cd* __restrict__ Qq,
                              cd* __restrict__ RPN, cd* __restrict__ RNEW) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (j >= n) return;
  const int a = r / n, i = r - a * n;
  const size_t o = (size_t)r * ld + j;
  const cd m = mval(W, D, a, i, j, ld);
  const cd m2 = R2[o];
  const cd m3 = T[o] + m2 * D[(size_t)a * ld + j];
  const double cq0 = 1.0 / 6, cq1 = 1.0 / 120, cq2 = 1.0 / 5040, cr0 = 0.5, cr1 = -1.0 / 24,
               cr2 = 1.0 / 240;
  const double h3 = h * h * h, h5 = h3 * h * h, h7 = h5 * h * h;
  cd q = (h3 * cq0) * m + (h5 * cq1) * m2 + (h7 * cq2) * m3;
  if (i == j) q = q + cd{h, 0.0};
  const cd rr = (h * cr0) * m + (h3 * cr1) * m2 + (h5 * cr2) * m3;
  Qq[o] = q;
  RNEW[o] = rr;
  cd rpn = RP[o] + rr;
  if (D13) {
    const size_t os = (size_t)i * ld + j;
    rpn = RP[o] + rr - c0dz * D13[os] + M3s[os];
  }
  RPN[o] = rpn;
}

// rp <- r + c0 dz D13 + M3s (end of an m6 slice, surf_magnus.f90:318).
__global__ void k_magnus6_carry(const cd* __restrict__ RNEW, const cd* __restrict__ D13,
                                const cd* __restrict__ M3s, double c0dz, int n, int ld,
                                cd* __restrict__ RP) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (j >= n) return;
  const int i = r % n;
  const size_t o = (size_t)r * ld + j, os = (size_t)i * ld + j;
  RP[o] = RNEW[o] + c0dz * D13[os] + M3s[os];
}

// M3s <- cm M3s + c1dz S13 (after M3s = D13 D13 by GEMM): m3 = c2 dz^3 m1 m1 + c1 dz q.
__global__ void k_magnus6_m3(cd* __restrict__ M3s, const cd* __restrict__ S13, double cm,
                             double c1dz, int n, int ld) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (j >= n) return;
  const size_t o = (size_t)i * ld + j;
  M3s[o] = cm * M3s[o] + c1dz * S13[o];
}

// A <- A + B (per angle, n x n block).
__global__ void k_add(cd* __restrict__ A, const cd* __restrict__ B, int n, int ld) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (j >= n) return;
  const size_t o = (size_t)r * ld + j;
  A[o] = A[o] + B[o];
}

dim3 grid_rows(int n, int rows) { return dim3(ceil_div(n, 128), rows); }

}  // namespace

void launch_magnus4_step(const cd* Vc, const cd* S, const cd* V1, const cd* V3, const cd* D,
                         int nang, int n, int ld, double h, double dz, double c0, double c1,
                         cd* Qq, cd* RPN, cd* RP, cudaStream_t st) {
  k_magnus4_step<<<grid_rows(n, nang * n), 128, 0, st>>>(Vc, S, V1, V3, D, n, ld, h, dz, c0, c1,
                                                         Qq, RPN, RP);
}
void launch_magnus6_shared(const cd* V1, const cd* V2, const cd* V3, int n, int ld, double d0,
                           double d1, cd* D13, cd* S13, cd* Wm, cd* Wp, cudaStream_t st) {
  k_magnus6_shared<<<grid_rows(n, n), 128, 0, st>>>(V1, V2, V3, n, ld, d0, d1, D13, S13, Wm, Wp);
}
void launch_magnus_square(const cd* S, const cd* W, const cd* D, int nang, int n, int ld, cd* R2,
                          cudaStream_t st) {
  k_magnus_square<<<grid_rows(n, nang * n), 128, 0, st>>>(S, W, D, n, ld, R2);
}
void launch_magnus6_exp(const cd* W, const cd* D, const cd* R2, const cd* T, int nang, int n,
                        int ld, double h, const cd* RP, const cd* D13, const cd* M3s, double c0dz,
                        cd* Qq, cd* RPN, cd* RNEW, cudaStream_t st) {
  k_magnus6_exp<<<grid_rows(n, nang * n), 128, 0, st>>>(W, D, R2, T, n, ld, h, RP, D13, M3s, c0dz,
                                                        Qq, RPN, RNEW);
}
void launch_magnus6_carry(const cd* RNEW, const cd* D13, const cd* M3s, double c0dz, int nang,
                          int n, int ld, cd* RP, cudaStream_t st) {
  k_magnus6_carry<<<grid_rows(n, nang * n), 128, 0, st>>>(RNEW, D13, M3s, c0dz, n, ld, RP);
}
void launch_magnus6_m3(cd* M3s, const cd* S13, double cm, double c1dz, int n, int ld,
                       cudaStream_t st) {
  k_magnus6_m3<<<grid_rows(n, n), 128, 0, st>>>(M3s, S13, cm, c1dz, n, ld);
}
void launch_add(cd* A, const cd* B, int nang, int n, int ld, cudaStream_t st) {
  k_add<<<grid_rows(n, nang * n), 128, 0, st>>>(A, B, n, ld);
}

}  // namespace trhepd
