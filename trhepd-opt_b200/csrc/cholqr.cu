// RK4 with CholeskyQR re-orthogonalisation (int_method 8): the boundary
// transforms of that method, the power estimate that triggers the
// re-orthogonalisation and the CholeskyQR itself, batched over angles with
// per-angle flags (sim-trhepd-rheed/src/surf_rk.f90:93-156, matcomp.f90:89-137,
// 530-594, matgs.f90:5-35).
#include <cuda_runtime.h>

#include "bulk.h"
#include "cholqr.h"
#include "launch_attr.h"

namespace trhepd {

namespace {

__device__ __forceinline__ cd conj_mul(cd a, cd b) {  // conj(a) b
  return cd{a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x};
}

// Sums of three doubles over the block (blockDim.x = kPeThreads); every thread
// receives the totals.
constexpr int kPeThreads = 256;
__device__ void block_sum3(double& a, double& b, double& c, double (*sh)[kPeThreads / 32]) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) {
    sh[0][warp] = a;
    sh[1][warp] = b;
    sh[2][warp] = c;
  }
  __syncthreads();
  a = b = c = 0.0;
  for (int w = 0; w < kPeThreads / 32; ++w) {
    a += sh[0][w];
    b += sh[1][w];
    c += sh[2][w];
  }
}

}  // namespace

// ---------------------------------------------------------------- boundary transforms
__global__ void k_invstrans_build(const cd* __restrict__ F, cd* __restrict__ Q,
                                  cd* __restrict__ P, const cd* __restrict__ gam, int n, int ld) {
  const int j = blockIdx.y * blockDim.x + threadIdx.x;
  const int r = blockIdx.x;
  if (j >= n) return;
  const int a = r / n, i = r - a * n;
  const cd fh = conj(F[((size_t)a * n + j) * n + i]);  // F^H(i,j) = conj(F(j,i))
  // q(j,i) = (delta + f(j,i)) / g_j, p(j,i) = i f(j,i) - i delta; Q = q^H, P = p^H
  const cd igc = conj(cdiv(cd{1.0, 0.0}, gam[(size_t)a * n + j]));
  const cd e = (i == j) ? cd{1.0 + fh.x, fh.y} : fh;
  const size_t o = (size_t)r * ld + j;
  Q[o] = e * igc;
  P[o] = (i == j) ? cd{0.0, 1.0} * cd{1.0 - fh.x, -fh.y} : cd{0.0, 1.0} * (-fh);
}

void launch_invstrans_build(const cd* F, cd* Q, cd* P, const cd* gam, int nang, int n, int ld,
                            cudaStream_t st) {
  dim3 grid(nang * n, ceil_div(n, 128));
  k_invstrans_build<<<grid, 128, 0, st>>>(F, Q, P, gam, n, ld);
}

__global__ void k_strans_build(cd* __restrict__ Q, cd* __restrict__ P, const cd* __restrict__ gam,
                               int n, int ld) {
  const int j = blockIdx.y * blockDim.x + threadIdx.x;
  const int r = blockIdx.x;
  if (j >= n) return;
  const int a = r / n;
  const size_t o = (size_t)r * ld + j;
  // q'(j,i) = g_j q(j,i) + i p(j,i), p'(j,i) = g_j q(j,i) - i p(j,i), conjugated
  const cd gx = Q[o] * conj(gam[(size_t)a * n + j]);
  const cd iy = cd{0.0, 1.0} * P[o];
  Q[o] = gx - iy;
  P[o] = gx + iy;
}

void launch_strans_build(cd* Q, cd* P, const cd* gam, int nang, int n, int ld, cudaStream_t st) {
  dim3 grid(nang * n, ceil_div(n, 128));
  k_strans_build<<<grid, 128, 0, st>>>(Q, P, gam, n, ld);
}

// ---------------------------------------------------------------- power estimate
// One block per angle; x, y = q x, y2 = p x and z = q^H y + p^H y2 in shared memory
// (in the stacked layout q x = Q^H x and q^H y = Q y).
__global__ void __launch_bounds__(kPeThreads) k_power_est(const cd* __restrict__ Q,
                                                           const cd* __restrict__ P,
                                                           cd* __restrict__ X, int* flag,
                                                           double* dval, int n, int ld,
                                                           int steps) {
  const int a = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  cd* Xa = X + (size_t)a * n;
  if (steps < 0) {
    const double s = 1.0 / sqrt(2.0 * n);
    for (int i = tid; i < n; i += kPeThreads) Xa[i] = cd{s, s};
    if (tid == 0) {
      flag[a] = 1;
      dval[a] = -1.0;
    }
    return;
  }
  extern __shared__ __align__(16) unsigned char pe_dyn[];
  cd* x = reinterpret_cast<cd*>(pe_dyn);
  cd* y = x + n;
  cd* y2 = y + n;
  cd* z = y2 + n;
  __shared__ double red[3][kPeThreads / 32];
  const cd* Qa = Q + (size_t)a * n * ld;
  const cd* Pa = P + (size_t)a * n * ld;
  for (int i = tid; i < n; i += kPeThreads) x[i] = Xa[i];
  __syncthreads();
  double d0 = -1.0, d = 0.0;
  for (int it = 0; it < steps; ++it) {
    for (int i = tid; i < n; i += kPeThreads) {
      cd s1 = cd{0.0, 0.0}, s2 = cd{0.0, 0.0};
      for (int j = 0; j < n; ++j) {
        s1 = s1 + conj_mul(Qa[(size_t)j * ld + i], x[j]);
        s2 = s2 + conj_mul(Pa[(size_t)j * ld + i], x[j]);
      }
      y[i] = s1;
      y2[i] = s2;
    }
    __syncthreads();
    for (int j = warp; j < n; j += kPeThreads / 32) {
      cd s = cd{0.0, 0.0};
      for (int i = lane; i < n; i += 32) s = s + Qa[(size_t)j * ld + i] * y[i];
      for (int i = lane; i < n; i += 32) s = s + Pa[(size_t)j * ld + i] * y2[i];
      for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
      }
      if (lane == 0) z[j] = s;
    }
    __syncthreads();
    double crx = 0.0, cry = 0.0, dn = 0.0;
    for (int i = tid; i < n; i += kPeThreads) {
      const cd c = z[i];
      dn += c.x * c.x + c.y * c.y;
      const cd t = conj_mul(x[i], c);
      crx += t.x;
      cry += t.y;
    }
    block_sum3(crx, cry, dn, red);
    d = hypot(crx, cry);
    const double inv = 1.0 / sqrt(dn);
    double dp = 0.0, u0 = 0.0, u1 = 0.0;
    for (int i = tid; i < n; i += kPeThreads) {
      const cd zi = cd{z[i].x * inv, z[i].y * inv};
      const cd c = zi - x[i];
      dp += c.x * c.x + c.y * c.y;
      x[i] = zi;
    }
    block_sum3(dp, u0, u1, red);  // also orders the x updates before the next step
    dp = sqrt(dp);
    if (dp < 1e-2 || d - d0 < 1e-2 * d) break;
    d0 = d;
  }
  for (int i = tid; i < n; i += kPeThreads) Xa[i] = x[i];
  if (tid == 0) {
    dval[a] = d;
    flag[a] = d > 1e2 ? 1 : 0;
  }
}

void launch_power_est(const cd* Q, const cd* P, cd* x, int* flag, double* dval, int nang, int n,
                      int ld, int steps, cudaStream_t st) {
  const size_t smem = (size_t)4 * n * sizeof(cd);
  static SmemOptIn attr;
  attr.ensure((const void*)k_power_est, smem);
  k_power_est<<<nang, kPeThreads, steps < 0 ? 0 : smem, st>>>(Q, P, x, flag, dval, n, ld, steps);
}

// ---------------------------------------------------------------- CholeskyQR
// T = S^H per flagged angle (n x n blocks, row stride ld), through 32 x 33 tiles.
__global__ void k_conj_transpose(const cd* __restrict__ S, cd* __restrict__ T,
                                 const int* __restrict__ flag, int n, int ld) {
  const int a = blockIdx.z;
  if (flag && !flag[a]) return;
  __shared__ cd tile[32][33];
  const cd* Sa = S + (size_t)a * n * ld;
  cd* Ta = T + (size_t)a * n * ld;
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
    const int r = e / 32, c = e % 32;
    if (r0 + r < n && c0 + c < n) tile[r][c] = Sa[(size_t)(r0 + r) * ld + c0 + c];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
    const int c = e / 32, r = e % 32;
    if (r0 + r < n && c0 + c < n) Ta[(size_t)(c0 + c) * ld + r0 + r] = conj(tile[r][c]);
  }
}

// Columns j0..j0+w-1 of the lower Cholesky factor of G (rows j0..n-1, the trailing
// matrix already updated): one block per flagged angle, the panel in shared
// memory, column by column.  Writes the factor back into G and its rows below the
// diagonal block, conjugate-transposed, into T (w x (n - j0 - w), row stride ld).
constexpr int kChThreads = 256;
__global__ void __launch_bounds__(kChThreads) k_chol_panel(cd* __restrict__ G, cd* __restrict__ T,
                                                           const int* __restrict__ flag, int n,
                                                           int ld, int j0, int w,
                                                           unsigned* status) {
  const int a = blockIdx.x;
  if (flag && !flag[a]) return;
  extern __shared__ __align__(16) unsigned char ch_dyn[];
  cd* S = reinterpret_cast<cd*>(ch_dyn);  // (n - j0) x 16
  __shared__ double inv;
  const int m = n - j0, tid = threadIdx.x;
  cd* Ga = G + (size_t)a * n * ld;
  for (int e = tid; e < m * 16; e += kChThreads) {
    const int i = e / 16, k = e % 16;
    S[e] = k < w ? Ga[(size_t)(j0 + i) * ld + j0 + k] : cd{0.0, 0.0};
  }
  __syncthreads();
  for (int jj = 0; jj < w; ++jj) {
    if (tid == 0) {
      double dd = S[jj * 16 + jj].x;
      if (!(dd > 0.0)) {
        atomicOr(status, kStatusZeroPivot);
        dd = fabs(dd) > 0.0 ? fabs(dd) : 1.0;
      }
      const double l = sqrt(dd);
      S[jj * 16 + jj] = cd{l, 0.0};
      inv = 1.0 / l;
    }
    __syncthreads();
    for (int i = jj + 1 + tid; i < m; i += kChThreads) S[i * 16 + jj] = inv * S[i * 16 + jj];
    __syncthreads();
    for (int e = tid; e < (m - jj - 1) * 16; e += kChThreads) {
      const int i = jj + 1 + e / 16, k = e % 16;
      if (k > jj && k < w && k <= i)
        S[i * 16 + k] = S[i * 16 + k] - S[i * 16 + jj] * conj(S[k * 16 + jj]);
    }
    __syncthreads();
  }
  cd* Ta = T + (size_t)a * n * ld;
  for (int e = tid; e < m * 16; e += kChThreads) {
    const int i = e / 16, k = e % 16;
    if (k < w && k <= i) Ga[(size_t)(j0 + i) * ld + j0 + k] = S[e];
    if (k < w && i >= w) Ta[(size_t)k * ld + (i - w)] = conj(S[e]);
  }
}

// Rows j0..j0+w-1 of X = L^{-1} [Q | P] (the rows above already solved, the ones
// from j0 on already reduced by them): one thread per column of [Q | P].
__global__ void k_trsv_block(cd* __restrict__ Q, cd* __restrict__ P, const cd* __restrict__ G,
                             const int* __restrict__ flag, int n, int ld, int j0, int w) {
  const int a = blockIdx.y;
  if (flag && !flag[a]) return;
  __shared__ cd Lb[16][16];
  const cd* Ga = G + (size_t)a * n * ld;
  for (int e = threadIdx.x; e < 256; e += blockDim.x) {
    const int i = e / 16, k = e % 16;
    Lb[i][k] = (i < w && k <= i) ? Ga[(size_t)(j0 + i) * ld + j0 + k] : cd{0.0, 0.0};
  }
  __syncthreads();
  const int vc = blockIdx.x * blockDim.x + threadIdx.x;
  if (vc >= 2 * n) return;
  cd* base = (vc < n ? Q + vc : P + (vc - n)) + (size_t)a * n * ld + (size_t)j0 * ld;
  cd x[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if (k < w) {
      cd s = base[(size_t)k * ld];
#pragma unroll
      for (int mm = 0; mm < 16; ++mm)
        if (mm < k) s = s - Lb[k][mm] * x[mm];
      x[k] = (1.0 / Lb[k][k].x) * s;
      base[(size_t)k * ld] = x[k];
    } else {
      x[k] = cd{0.0, 0.0};
    }
  }
}

size_t cholqr_scratch_bytes(int nang, int n, int ld) {
  return 2 * (size_t)nang * n * ld * sizeof(cd) + 256;
}

static void masked_gemm(const cd* A, const cd* B, cd* Cm, int M, int N, int K, int ld,
                        long long stride, double alpha, int beta, int nang, const int* flag,
                        cudaStream_t st) {
  BatchedGemm g{A, B, Cm, M, N, K, ld, ld, ld, stride, stride, stride, cd{alpha, 0.0}, beta,
                nang, flag};
  launch_zgemm_batched(g, st);
}

int launch_cholqr(cd* Q, cd* P, const int* flag, int nang, int n, int ld, void* scratch,
                  unsigned* status, cudaStream_t st) {
  cd* G = reinterpret_cast<cd*>(scratch);
  cd* T = G + (size_t)nang * n * ld;
  const long long sa = (long long)n * ld;
  int launches = 0;
  // G = Q Q^H + P P^H
  dim3 tg(ceil_div(n, 32), ceil_div(n, 32), nang);
  k_conj_transpose<<<tg, 256, 0, st>>>(Q, T, flag, n, ld);
  masked_gemm(Q, T, G, n, n, n, ld, sa, 1.0, 0, nang, flag, st);
  k_conj_transpose<<<tg, 256, 0, st>>>(P, T, flag, n, ld);
  masked_gemm(P, T, G, n, n, n, ld, sa, 1.0, 1, nang, flag, st);
  launches += 4;
  // G = L L^H, right-looking in 16-column panels
  static SmemOptIn attr;
  attr.ensure((const void*)k_chol_panel, (size_t)n * 16 * sizeof(cd));
  for (int j0 = 0; j0 < n; j0 += 16) {
    const int w = n - j0 < 16 ? n - j0 : 16, rest = n - j0 - w;
    k_chol_panel<<<nang, kChThreads, (size_t)(n - j0) * 16 * sizeof(cd), st>>>(G, T, flag, n, ld,
                                                                               j0, w, status);
    ++launches;
    if (rest > 0) {
      cd* G22 = G + (size_t)(j0 + w) * ld + (j0 + w);
      masked_gemm(G + (size_t)(j0 + w) * ld + j0, T, G22, rest, rest, w, ld, sa, -1.0, 1, nang,
                  flag, st);
      ++launches;
    }
  }
  // [Q | P] <- L^{-1} [Q | P], block forward substitution
  for (int j0 = 0; j0 < n; j0 += 16) {
    const int w = n - j0 < 16 ? n - j0 : 16, rest = n - j0 - w;
    dim3 grid(ceil_div(2 * n, 128), nang);
    k_trsv_block<<<grid, 128, 0, st>>>(Q, P, G, flag, n, ld, j0, w);
    ++launches;
    if (rest > 0) {
      const cd* L21 = G + (size_t)(j0 + w) * ld + j0;
      masked_gemm(L21, Q + (size_t)j0 * ld, Q + (size_t)(j0 + w) * ld, rest, n, w, ld, sa, -1.0,
                  1, nang, flag, st);
      masked_gemm(L21, P + (size_t)j0 * ld, P + (size_t)(j0 + w) * ld, rest, n, w, ld, sa, -1.0,
                  1, nang, flag, st);
      launches += 2;
    }
  }
  return launches;
}

}  // namespace trhepd
