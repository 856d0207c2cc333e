// Bulk reflection matrices on the GPU: blkref (sim-trhepd-rheed/src/bulk.f90:7-128)
// for every (angle, beam group) at once.
//
// The reference forms each slice's transfer matrix from the eigendecomposition
// of the slice Hamiltonian H (trmatg.f90:6-59):
//     T = [tau e, rho e^-1; rho e, tau e^-1] [tau rho; rho tau]^-1,
//     tau = (gamma_i + kappa_j) u_ij,  rho = (gamma_i - kappa_j) u_ij.
// With w = (psi, psi') and c = S w, S = [G, -iI; G, iI] (G = diag gamma), the
// right factor maps mode amplitudes to c and the left one advances them by dz, so
//     T = S exp(dz [0 I; -H 0]) S^-1,
//     exp(dz [0 I; -H 0]) = [C, s; -H s, C],  C = cos(sqrt(H) dz),
//                                               s = sin(sqrt(H) dz)/sqrt(H).
// C and s come from a degree-8 Taylor series in X = -H h^2 on h = dz / 2^m
// (||X|| <= 1/4) followed by m double-angle steps C <- 2C^2 - I, s <- 2 s C:
// batched complex GEMMs, no eigensolver.  Each slice's propagator is converted
// to mode space and the slices are chained there, as the reference chains its
// slice transfer matrices (bulk.f90:67-79): chaining in w-space and converting
// once would form the decaying blocks of strongly evanescent beams (e^{-kappa c},
// ~1e-20 over a layer) as differences of ~1e20 entries.  Then the layer
// recursion R <- (T12 + T11 R)(T22 + T21 R)^-1 with the reference's convergence
// exit (bulk.f90:95-119).
#include <cuda_runtime.h>

#include <cmath>

#include "bulk.h"
#include "kernels.h"
#include "launch_attr.h"

namespace trhepd {

// ============================================================ batched complex GEMM
// C_b = alpha A_b B_b + beta C_b (row-major, FP64 DMMA), beta in {0, 1}.
namespace bgemm {
constexpr int BM = 64, BN = 64, BK = 16, STAGES = 3;
constexpr int ASTR = BK + 4, BSTR = BN + 2;
constexpr int A_TILE = BM * ASTR, B_TILE = BK * BSTR;
constexpr size_t SMEM = (size_t)STAGES * (A_TILE + B_TILE) * sizeof(cd);
}  // namespace bgemm

__device__ __forceinline__ void b_cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void b_dmma(double& c0, double& c1, double& c2, double& c3, double a0,
                                       double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
      : "d"(a0), "d"(a1), "d"(b0));
}

__global__ void __launch_bounds__(128, 2)
    k_zgemm_batched(BatchedGemm g) {
  using namespace bgemm;
  const int b = blockIdx.z;
  if (g.active && !g.active[b]) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* As = reinterpret_cast<cd*>(smem_raw);
  cd* Bs = As + STAGES * A_TILE;
  const cd* A = g.A + (size_t)b * g.sA;
  const cd* B = g.B + (size_t)b * g.sB;
  cd* C = g.C + (size_t)b * g.sC;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, t = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int bm = blockIdx.y * BM, bn = blockIdx.x * BN;
  auto load_stage = [&](int s, int k0) {
    cd* a = As + s * A_TILE;
    cd* bb = Bs + s * B_TILE;
#pragma unroll
    for (int it = 0; it < (BM * BK) / 128; ++it) {
      int e = tid + it * 128;
      int r = e / BK, kk = e % BK;
      bool ok = bm + r < g.M && k0 + kk < g.K;
      b_cp_async16(a + r * ASTR + kk, ok ? A + (size_t)(bm + r) * g.lda + k0 + kk : A, ok);
    }
#pragma unroll
    for (int it = 0; it < (BK * BN) / 128; ++it) {
      int e = tid + it * 128;
      int kk = e / BN, c = e % BN;
      bool ok = k0 + kk < g.K && bn + c < g.N;
      b_cp_async16(bb + kk * BSTR + c, ok ? B + (size_t)(k0 + kk) * g.ldb + bn + c : B, ok);
    }
  };
  double cr[2][4][4], ci[2][4][4];
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) cr[mi][ni][e] = ci[mi][ni][e] = 0.0;
  const int nk = (g.K + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load_stage(s, s * BK);
    asm volatile("cp.async.commit_group;\n" ::);
  }
  for (int kt = 0; kt < nk; ++kt) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 2));
    __syncthreads();
    int nxt = kt + STAGES - 1;
    if (nxt < nk) load_stage(nxt % STAGES, nxt * BK);
    asm volatile("cp.async.commit_group;\n" ::);
    const cd* a = As + (kt % STAGES) * A_TILE;
    const cd* bb = Bs + (kt % STAGES) * B_TILE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      cd af[2][2], bf[4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        af[mi][0] = a[(wm + mi * 16 + gq) * ASTR + kk + t];
        af[mi][1] = a[(wm + mi * 16 + gq + 8) * ASTR + kk + t];
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = bb[(kk + t) * BSTR + wn + ni * 8 + gq];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          double* R = cr[mi][ni];
          double* I = ci[mi][ni];
          b_dmma(R[0], R[1], R[2], R[3], af[mi][0].x, af[mi][1].x, bf[ni].x);
          b_dmma(R[0], R[1], R[2], R[3], -af[mi][0].y, -af[mi][1].y, bf[ni].y);
          b_dmma(I[0], I[1], I[2], I[3], af[mi][0].x, af[mi][1].x, bf[ni].y);
          b_dmma(I[0], I[1], I[2], I[3], af[mi][0].y, af[mi][1].y, bf[ni].x);
        }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int r = bm + wm + mi * 16 + gq + ((e >= 2) ? 8 : 0);
        int c = bn + wn + ni * 8 + 2 * t + (e & 1);
        if (r < g.M && c < g.N) {
          cd v = g.alpha * cd{cr[mi][ni][e], ci[mi][ni][e]};
          size_t o = (size_t)r * g.ldc + c;
          C[o] = g.beta ? C[o] + v : v;
        }
      }
}

void launch_zgemm_batched(const BatchedGemm& g, cudaStream_t st) {
  using namespace bgemm;
  static SmemOptIn attr;
  attr.ensure((const void*)k_zgemm_batched, SMEM);
  dim3 grid(ceil_div(g.N, BN), ceil_div(g.M, BM), g.batch);
  k_zgemm_batched<<<grid, 128, SMEM, st>>>(g);
}

// ============================================================ bulk element kernels
// X = -H h^2 with H = V(slice) + diag(gamma^2) for item b (angle, group), padded to n.
// H(i,i) = u0 + g_i^2; H(j,i) = u(e) (j > i); H(i,j) = conj(w(e)), e = iv(j,i)
// (trmatg.f90:150-157).  Also keeps H for the -H s term.
__global__ void k_bulk_hamiltonian(const TableEntry* __restrict__ tcol, const int* __restrict__ pair,
                                   const cd* __restrict__ gam, const int* __restrict__ gsize,
                                   int ngr, int n, int ld, double h2, cd* __restrict__ H,
                                   cd* __restrict__ X) {
  const int b = blockIdx.y;
  const int grp = b % ngr;
  const int m = gsize[grp];
  const int* pg = pair + (size_t)grp * n * n;  // symmetric: iv(max, min) - 1 of the group
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += gridDim.x * blockDim.x) {
    int i = e / n, j = e % n;
    cd v = cd{0.0, 0.0};
    if (i < m && j < m) {
      if (i == j) {
        cd g = gam[(size_t)b * n + i];
        v = tcol[0].u + g * g;
      } else if (i > j) {  // H(i, j), i > j: u(iv(i, j))
        v = tcol[pg[j * n + i]].u;
      } else {             // H(i, j), i < j: conj(w(iv(j, i)))
        v = conj(tcol[pg[i * n + j]].w);
      }
    }
    size_t o = ((size_t)b * n + i) * ld + j;
    H[o] = v;
    X[o] = -h2 * v;
  }
}

// out = c0 I + c1 X + c2 X2 + c3 X3 + c4 X4 (X4 may be null)
__global__ void k_bulk_poly(const cd* __restrict__ X, const cd* __restrict__ X2,
                            const cd* __restrict__ X3, const cd* __restrict__ X4, double c0,
                            double c1, double c2, double c3, double c4, int n, int ld, int batch,
                            cd* __restrict__ out) {
  size_t total = (size_t)batch * n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t b = e / ((size_t)n * n);
    int r = (int)(e % ((size_t)n * n));
    int i = r / n, j = r % n;
    size_t o = (b * n + i) * ld + j;
    cd v = c1 * X[o] + c2 * X2[o] + c3 * X3[o];
    if (X4) v = v + c4 * X4[o];
    if (i == j) v.x += c0;
    out[o] = v;
  }
}

// A <- alpha * A + beta * B (+ gamma on the diagonal)
__global__ void k_bulk_axpby(cd* __restrict__ A, const cd* __restrict__ B, double alpha,
                             double beta, double diag, int n, int ld, int batch) {
  size_t total = (size_t)batch * n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t b = e / ((size_t)n * n);
    int r = (int)(e % ((size_t)n * n));
    int i = r / n, j = r % n;
    size_t o = (b * n + i) * ld + j;
    cd v = alpha * A[o] + (B ? beta * B[o] : cd{0.0, 0.0});
    if (i == j) v.x += diag;
    A[o] = v;
  }
}

// E = [C, s; -Hs, C] (2n x 2n, ld2)
__global__ void k_bulk_build_e(const cd* __restrict__ C, const cd* __restrict__ S,
                               const cd* __restrict__ Hs, int n, int ld, int ld2, int batch,
                               cd* __restrict__ E) {
  size_t total = (size_t)batch * n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t b = e / ((size_t)n * n);
    int r = (int)(e % ((size_t)n * n));
    int i = r / n, j = r % n;
    size_t o = (b * n + i) * ld + j;
    cd* Eb = E + b * 2 * n * ld2;
    Eb[(size_t)i * ld2 + j] = C[o];
    Eb[(size_t)i * ld2 + n + j] = S[o];
    Eb[(size_t)(n + i) * ld2 + j] = -Hs[o];
    Eb[(size_t)(n + i) * ld2 + n + j] = C[o];
  }
}

// T = S E S^-1 (see file header), times the unit-layer phase shift of columns
// j, j+n (bulk.f90:83-93) when `phase` is given; padded beams use gamma = 1.
__global__ void k_bulk_similarity(const cd* __restrict__ E, const cd* __restrict__ gam,
                                  const cd* __restrict__ phase, const int* __restrict__ gsize,
                                  int ngr, int n, int ld2, int batch, cd* __restrict__ T) {
  size_t total = (size_t)batch * n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t b = e / ((size_t)n * n);
    int r = (int)(e % ((size_t)n * n));
    int i = r / n, j = r % n;
    const int m = gsize[b % ngr];
    const cd* Eb = E + b * 2 * n * ld2;
    cd gi = (i < m) ? gam[b * n + i] : cd{1.0, 0.0};
    cd gj = (j < m) ? gam[b * n + j] : cd{1.0, 0.0};
    cd e11 = Eb[(size_t)i * ld2 + j], e12 = Eb[(size_t)i * ld2 + n + j];
    cd e21 = Eb[(size_t)(n + i) * ld2 + j], e22 = Eb[(size_t)(n + i) * ld2 + n + j];
    const cd I = cd{0.0, 1.0};
    cd A = gi * e11 - I * e21, B = gi * e12 - I * e22;
    cd Cc = gi * e11 + I * e21, D = gi * e12 + I * e22;
    cd ig = cdiv(cd{1.0, 0.0}, gj);
    cd ph = (phase && j < m) ? phase[b * n + j] : cd{1.0, 0.0};
    cd* Tb = T + b * 2 * n * ld2;
    Tb[(size_t)i * ld2 + j] = ph * (0.5 * (A * ig + I * B));
    Tb[(size_t)i * ld2 + n + j] = ph * (0.5 * (A * ig - I * B));
    Tb[(size_t)(n + i) * ld2 + j] = ph * (0.5 * (Cc * ig + I * D));
    Tb[(size_t)(n + i) * ld2 + n + j] = ph * (0.5 * (Cc * ig - I * D));
  }
}

// Unit-layer phase shift (bulk.f90:83-93): columns j and j+n of T times ph_j.
__global__ void k_bulk_phase_cols(cd* __restrict__ T, const cd* __restrict__ phase,
                                  const int* __restrict__ gsize, int ngr, int n, int ld2,
                                  int batch) {
  size_t total = (size_t)batch * 2 * n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t b = e / ((size_t)2 * n * n);
    int r = (int)(e % ((size_t)2 * n * n));
    int i = r / n, j = r % n;
    if (j >= gsize[b % ngr]) continue;
    const cd ph = phase[b * n + j];
    cd* Tb = T + b * 2 * n * ld2 + (size_t)i * ld2;
    Tb[j] = ph * Tb[j];
    Tb[n + j] = ph * Tb[n + j];
  }
}

// t1 = T12, t2 = T22 (first layer), for active items
__global__ void k_bulk_layer_init(const cd* __restrict__ T, const int* __restrict__ active, int n,
                                  int ld, int ld2, int batch, cd* __restrict__ t1,
                                  cd* __restrict__ t2) {
  size_t total = (size_t)batch * n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t b = e / ((size_t)n * n);
    if (!active[b]) continue;
    int r = (int)(e % ((size_t)n * n));
    int i = r / n, j = r % n;
    const cd* Tb = T + b * 2 * n * ld2;
    t1[(b * n + i) * ld + j] = Tb[(size_t)i * ld2 + n + j];
    t2[(b * n + i) * ld + j] = Tb[(size_t)(n + i) * ld2 + n + j];
  }
}

// Q = t2^T, P = t1^T (right division through the left solve); padded beams get
// an identity block so the solve stays regular.
__global__ void k_bulk_transpose_pair(const cd* __restrict__ t1, const cd* __restrict__ t2,
                                      const int* __restrict__ active, const int* __restrict__ gsize,
                                      int ngr, int n, int ld, int batch, cd* __restrict__ Q,
                                      cd* __restrict__ P) {
  size_t total = (size_t)batch * n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    size_t b = e / ((size_t)n * n);
    if (!active[b]) continue;
    int r = (int)(e % ((size_t)n * n));
    int i = r / n, j = r % n;
    const int m = gsize[b % ngr];
    size_t o = (b * n + i) * ld + j, ot = (b * n + j) * ld + i;
    if (i < m && j < m) {
      Q[o] = t2[ot];
      P[o] = t1[ot];
    } else {
      Q[o] = cd{(i == j) ? 1.0 : 0.0, 0.0};
      P[o] = cd{0.0, 0.0};
    }
  }
}

// R = P^T; convergence test of the reference (bulk.f90:105-118): at layer 20 keep
// |R_ii|^2, after it stop the item once max_i ||R_ii|^2 - previous| < epsb.
__global__ void k_bulk_layer_finish(const cd* __restrict__ P, int* __restrict__ active,
                                    const int* __restrict__ gsize, int ngr, int n, int ld,
                                    int layer, double epsb, double* __restrict__ r20,
                                    cd* __restrict__ R) {
  const int b = blockIdx.x;
  if (!active[b]) return;
  const int m = gsize[b % ngr];
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    int i = e / n, j = e % n;
    R[((size_t)b * n + i) * ld + j] = P[((size_t)b * n + j) * ld + i];
  }
  __syncthreads();
  if (layer < 20) return;
  __shared__ double red[32];
  double rmax = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    cd d = R[((size_t)b * n + i) * ld + i];
    double r2 = (d * conj(d)).x;
    if (layer > 20) rmax = fmax(rmax, fabs(r2 - r20[(size_t)b * n + i]));
    r20[(size_t)b * n + i] = r2;
  }
  for (int o = 16; o > 0; o >>= 1) rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) rmax = fmax(rmax, red[w]);
    if (layer > 20 && rmax < epsb) active[b] = 0;
  }
}

static int grid_for(size_t total) {
  size_t g = (total + 255) / 256;
  return (int)(g > 148 * 16 ? 148 * 16 : (g ? g : 1));
}

void launch_bulk_hamiltonian(const TableEntry* tcol, const int* pair, const cd* gam,
                             const int* gsize, int ngr, int n, int ld, int batch, double h2, cd* H,
                             cd* X, cudaStream_t st) {
  dim3 grid(ceil_div(n * n, 256), batch);
  k_bulk_hamiltonian<<<grid, 256, 0, st>>>(tcol, pair, gam, gsize, ngr, n, ld, h2, H, X);
}
void launch_bulk_poly(const cd* X, const cd* X2, const cd* X3, const cd* X4, const double* c,
                      int n, int ld, int batch, cd* out, cudaStream_t st) {
  size_t total = (size_t)batch * n * n;
  k_bulk_poly<<<grid_for(total), 256, 0, st>>>(X, X2, X3, X4, c[0], c[1], c[2], c[3], c[4], n, ld,
                                                batch, out);
}
void launch_bulk_axpby(cd* A, const cd* B, double alpha, double beta, double diag, int n, int ld,
                       int batch, cudaStream_t st) {
  size_t total = (size_t)batch * n * n;
  k_bulk_axpby<<<grid_for(total), 256, 0, st>>>(A, B, alpha, beta, diag, n, ld, batch);
}
void launch_bulk_build_e(const cd* C, const cd* S, const cd* Hs, int n, int ld, int ld2, int batch,
                         cd* E, cudaStream_t st) {
  size_t total = (size_t)batch * n * n;
  k_bulk_build_e<<<grid_for(total), 256, 0, st>>>(C, S, Hs, n, ld, ld2, batch, E);
}
void launch_bulk_similarity(const cd* E, const cd* gam, const cd* phase, const int* gsize, int ngr,
                            int n, int ld2, int batch, cd* T, cudaStream_t st) {
  size_t total = (size_t)batch * n * n;
  k_bulk_similarity<<<grid_for(total), 256, 0, st>>>(E, gam, phase, gsize, ngr, n, ld2, batch, T);
}
void launch_bulk_phase_cols(cd* T, const cd* phase, const int* gsize, int ngr, int n, int ld2,
                            int batch, cudaStream_t st) {
  size_t total = (size_t)batch * 2 * n * n;
  k_bulk_phase_cols<<<grid_for(total), 256, 0, st>>>(T, phase, gsize, ngr, n, ld2, batch);
}
void launch_bulk_layer_init(const cd* T, const int* active, int n, int ld, int ld2, int batch,
                            cd* t1, cd* t2, cudaStream_t st) {
  size_t total = (size_t)batch * n * n;
  k_bulk_layer_init<<<grid_for(total), 256, 0, st>>>(T, active, n, ld, ld2, batch, t1, t2);
}
void launch_bulk_transpose_pair(const cd* t1, const cd* t2, const int* active, const int* gsize,
                                int ngr, int n, int ld, int batch, cd* Q, cd* P,
                                cudaStream_t st) {
  size_t total = (size_t)batch * n * n;
  k_bulk_transpose_pair<<<grid_for(total), 256, 0, st>>>(t1, t2, active, gsize, ngr, n, ld, batch,
                                                          Q, P);
}
void launch_bulk_layer_finish(const cd* P, int* active, const int* gsize, int ngr, int n, int ld,
                              int batch, int layer, double epsb, double* r20, cd* R,
                              cudaStream_t st) {
  k_bulk_layer_finish<<<batch, 256, 0, st>>>(P, active, gsize, ngr, n, ld, layer, epsb, r20, R);
}

}  // namespace trhepd
