// FP64 kernels of the multislice surface solve (sm_100a).
//
//   K2 structure factors        strfac      sim-trhepd-rheed/src/strfac.f90:65-75
//   K3 stage potential table    scpot x3    scpot.f90:115-193, surfio.f90:29-41
//   K4 stage-matrix gather      vvi2mate    matcomp.f90:253-279
//   K5 stage GEMM + RKN update  hp_pinth/hp_qinth  surf_prkn.f90:222-276
//   K7 Gershgorin estimate      cond_est    matcomp.f90:498-528
//   K8 renormalisation Q^-1 P   matAbdivB   matcomp.f90:53-69
//   boundary transforms         invstransh/stransh  matcomp.f90:140-196
//   intensities                 surflf.f90:142-151
#include <cuda_runtime.h>

#include <cstdio>

#include "kernels.h"
#include "launch_attr.h"

namespace trhepd {

// ============================================================ K2 structure factors
// One thread per (k, atom); the <= 12 plane-group images are summed in registers.
__global__ void k_structure_factor(const double* __restrict__ gh, const double* __restrict__ gk,
                                   int nv, const double* __restrict__ img,
                                   const int* __restrict__ nimg, int natm, double dx, double dy,
                                   cd* __restrict__ st) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (k >= nv || j >= natm) return;
  double sr = 0.0, si = 0.0;
  int n = nimg[j];
  for (int m = 0; m < n; ++m) {
    double xb = img[(j * 12 + m) * 2], yb = img[(j * 12 + m) * 2 + 1];
    double gr = gh[k] * (dx + xb) + gk[k] * (dy + yb);
    double s, c;
    sincos(gr, &s, &c);
    sr += c;
    si += s;
  }
  st[(size_t)j * nv + k] = cd{sr, si};
}

void launch_structure_factor(const double* gh, const double* gk, int nv, const double* img,
                             const int* nimg, int natm, double dx, double dy, cd* st,
                             cudaStream_t stream) {
  if (natm <= 0 || nv <= 0) return;
  dim3 grid(ceil_div(nv, 128), natm);
  k_structure_factor<<<grid, 128, 0, stream>>>(gh, gk, nv, img, nimg, natm, dx, dy, st);
}

// ============================================================ K3 potential table
// Block per stage depth; the depth-dependent Gaussian factors exp(b (z - z_j)^2) of
// every (atom, Gaussian) are formed once in shared memory, then each thread sums
// the atoms for its Fourier components (coalesced over k).
constexpr int kMaxPotAtoms = 512;
constexpr int kMaxGauss = 6;

__global__ void k_potential_table(PotInputs in, const double* __restrict__ depth,
                                  TableEntry* __restrict__ table) {
  const int c = blockIdx.x;
  const double zc = depth[c];
  const double uf = -70.0;
  __shared__ double sE[kMaxPotAtoms * kMaxGauss];
  __shared__ double sZ1[kMaxPotAtoms];  // z1 = zi - z_j (needed by the ion term)
  __shared__ int sElem[kMaxPotAtoms];
  const int nabr = in.nabr, mab = in.mab, nv = in.nv;
  // flatten atoms of the three parts
  int base[4];
  base[0] = 0;
  for (int p = 0; p < 3; ++p) base[p + 1] = base[p] + in.part[p].natm;
  const int ntot = base[3];
  for (int t = threadIdx.x; t < ntot; t += blockDim.x) {
    int p = (t >= base[1]) + (t >= base[2]);
    int j = t - base[p];
    const PotPart& P = in.part[p];
    double zi = zc + P.zshift;
    double ocrmesh = P.rmesh * P.ocr[j];
    int ie = P.ielm[j];
    double z1 = zi - P.z[j];
    double z2 = z1 * z1;
    sZ1[t] = z1;
    sElem[t] = ie;
    for (int i = 0; i < nabr; ++i) {
      double ex = in.b[ie * mab + i] * z2;
      sE[t * kMaxGauss + i] = (ex > uf) ? exp(ex) * ocrmesh : 0.0;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nv; k += blockDim.x) {
    double vr = 0.0, vim = 0.0;  // v and vi accumulated separately
    double vir = 0.0, vii = 0.0;
    for (int p = 0; p < 3; ++p) {
      const PotPart& P = in.part[p];
      if (k >= P.nk) continue;
      for (int j = 0; j < P.natm; ++j) {
        int t = base[p] + j;
        int ie = sElem[t];
        double ocrmesh = P.rmesh * P.ocr[j];
        double tv = 0.0;
        if (fabs(in.dchg[ie]) > 1e-4) {  // ionic term (scpot.f90:139-150)
          double z1 = -fabs(sZ1[t]);
          if (k == 0) {
            tv = ocrmesh * z1 * in.dchg[ie];
          } else {
            double ex = in.ghk[k] * z1;
            tv = (ex > uf) ? exp(ex) * ocrmesh / in.ghk[k] * in.dchg[ie] : 0.0;
          }
        }
        double tvi = 0.0;
        const double* asf_e = in.asf + (size_t)ie * mab * nv;
        if (in.nabi == 1) {
          double sap = asf_e[(size_t)nabr * nv + 0];
          for (int i = 0; i < nabr; ++i) {
            double aex = asf_e[(size_t)i * nv + k] * sE[t * kMaxGauss + i];
            tv = tv + aex;
            tvi = tvi + fabs(sap * aex);
          }
        } else {
          for (int i = 0; i < nabr; ++i) tv = tv + asf_e[(size_t)i * nv + k] * sE[t * kMaxGauss + i];
        }
        cd ct = P.st[(size_t)j * P.nk + k];
        vr = vr + tv * ct.x;
        vim = vim + tv * ct.y;
        // vi += (0, tvi) * ct
        vir = vir + (0.0 * ct.x - tvi * ct.y);
        vii = vii + (0.0 * ct.y + tvi * ct.x);
      }
    }
    TableEntry e;
    e.u = cd{vr + vir, vim + vii};
    e.w = cd{vr - vir, vim - vii};
    table[(size_t)c * nv + k] = e;
  }
}

void launch_potential_table(const PotInputs& in, const double* depth, int ncol, TableEntry* table,
                            cudaStream_t st) {
  if (ncol <= 0) return;
  k_potential_table<<<ncol, 256, 0, st>>>(in, depth, table);
}

// ============================================================ K4 gather
__global__ void k_gather_stage(const TableEntry* __restrict__ tc, const int* __restrict__ pair,
                               int n, int kpad, int ld, int drop_diag, cd* __restrict__ V) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int k = blockIdx.y;
  if (j >= ld || k >= kpad) return;
  cd v = cd{0.0, 0.0};
  if (k < n && j < n) {
    if (k < j) {
      v = -conj(tc[pair[k * n + j]].u);
    } else if (k > j) {
      v = -tc[pair[k * n + j]].w;
    } else if (!drop_diag) {
      v = -conj(tc[0].u);
    }
  }
  V[(size_t)k * ld + j] = v;
  // with the diagonal dropped, its (constant) value is kept in the slot after the matrix
  if (drop_diag && k == 0 && j == 0) V[(size_t)kpad * ld] = -conj(tc[0].u);
}

// One stage matrix per problem of a stacked group: problem b gathers from its own
// table (tables[b] + coloff) into V + b * vstride.
__global__ void k_gather_stage_multi(const TableEntry* const* __restrict__ tables, size_t coloff,
                                     const int* __restrict__ pair, int n, int kpad, int ld,
                                     int drop_diag, cd* __restrict__ V, long long vstride) {
  const int b = blockIdx.z;
  const TableEntry* tc = tables[b] + coloff;
  cd* Vb = V + (size_t)b * vstride;
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int k = blockIdx.y;
  if (j >= ld || k >= kpad) return;
  cd v = cd{0.0, 0.0};
  if (k < n && j < n) {
    if (k < j) {
      v = -conj(tc[pair[k * n + j]].u);
    } else if (k > j) {
      v = -tc[pair[k * n + j]].w;
    } else if (!drop_diag) {
      v = -conj(tc[0].u);
    }
  }
  Vb[(size_t)k * ld + j] = v;
  if (drop_diag && k == 0 && j == 0) Vb[(size_t)kpad * ld] = -conj(tc[0].u);
}

void launch_gather_stage_multi(const TableEntry* const* tables, size_t coloff, const int* pair,
                               int n, int kpad, int ld, bool drop_diag, cd* V, long long vstride,
                               int nprob, cudaStream_t st) {
  dim3 grid(ceil_div(ld, 128), kpad, nprob);
  k_gather_stage_multi<<<grid, 128, 0, st>>>(tables, coloff, pair, n, kpad, ld, drop_diag ? 1 : 0,
                                             V, vstride);
}

void launch_gather_stage(const TableEntry* table_col, const int* pair, int n, int kpad, int ld,
                         bool drop_diag, cd* V, cudaStream_t st) {
  dim3 grid(ceil_div(ld, 128), kpad);
  k_gather_stage<<<grid, 128, 0, st>>>(table_col, pair, n, kpad, ld, drop_diag ? 1 : 0, V);
}

// ============================================================ identity-stage elementwise
__global__ void k_stage_identity(cd* __restrict__ Q, cd* __restrict__ P, const cd* __restrict__ V,
                                 const cd* __restrict__ D, int nang, int n, int ld, double cb,
                                 double ca, StackedRows sr) {
  int j = blockIdx.y * blockDim.x + threadIdx.x;
  int r = blockIdx.x;  // stacked row
  if (j >= n) return;
  int a = r / n, i = r - a * n;
  size_t o = (size_t)r * ld + j;
  if (sr.rows_b > 0) V += (size_t)(r / sr.rows_b) * sr.vstride;
  cd m = V[(size_t)i * ld + j];
  if (i == j) m = m + D[(size_t)a * ld + j];
  cd p = P[o] + cb * m;
  P[o] = p;
  cd q = ca * p;
  if (i == j) q.x += 1.0;
  Q[o] = q;
}

void launch_stage_identity(cd* Q, cd* P, const cd* V, const cd* D, int nang, int n, int ld,
                           double cb, double ca, cudaStream_t st, StackedRows sr) {
  dim3 grid(nang * n, ceil_div(n, 128));  // rows on x: more than 65535 stacked rows
  k_stage_identity<<<grid, 128, 0, st>>>(Q, P, V, D, nang, n, ld, cb, ca, sr);
}

// ============================================================ K5 FP64 DMMA stage GEMM
// CTA tile 64 x 64 complex, k-step 16, 4 warps (2 x 2), warp tile 32 x 32 built
// from m16n8k4 FP64 MMAs (4 real MMAs per complex product).  3-stage cp.async
// pipeline; shared-memory rows padded so fragment loads are conflict-free.
namespace f64gemm {
constexpr int BM = 64, BN = 64, BK = 16, STAGES = 3;
constexpr int ASTR = BK + 4;   // complex elements per A row in smem (stride = 4 mod 8 x 16B)
constexpr int BSTR = BN + 2;   // complex elements per B row in smem (stride = 2 mod 8 x 16B)
constexpr int A_TILE = BM * ASTR, B_TILE = BK * BSTR;
constexpr size_t SMEM = (size_t)STAGES * (A_TILE + B_TILE) * sizeof(cd);
}  // namespace f64gemm

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double& c2, double& c3, double a0,
                                     double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
      : "d"(a0), "d"(a1), "d"(b0));
}

__global__ void __launch_bounds__(128, 2)
    k_stage_gemm_f64(const cd* __restrict__ Q, cd* __restrict__ P, cd* __restrict__ Qo,
                     const cd* __restrict__ V, const cd* __restrict__ D, int rows, int n, int ld,
                     int kpad, double cb, double ca, StackedRows sr, int tiles_x, int ntiles) {
  using namespace f64gemm;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* As = reinterpret_cast<cd*>(smem_raw);
  cd* Bs = As + STAGES * A_TILE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int tpp = ceil_div(sr.rows_b, BM);
  const int rows_all = rows;
  const cd* const V_all = V;
  // one tile per block (a grid of every tile), or a capped grid whose blocks walk the
  // tiles (a context leaving SMs to other streams)
  const int stride = gridDim.x * gridDim.y;
  for (int tile = blockIdx.y * gridDim.x + blockIdx.x; tile < ntiles; tile += stride) {
  const int tx = tile % tiles_x, ty = tile / tiles_x;
  // row tile -> problem: tiles of one problem never take rows of the next
  const int pb = ty / tpp;
  const int bm = pb * sr.rows_b + (ty - pb * tpp) * BM, bn = tx * BN;
  rows = min(rows_all, (pb + 1) * sr.rows_b);
  V = V_all + (size_t)pb * sr.vstride;

  auto load_stage = [&](int s, int k0) {
    cd* a = As + s * A_TILE;
    cd* b = Bs + s * B_TILE;
#pragma unroll
    for (int it = 0; it < (BM * BK) / 128; ++it) {
      int e = tid + it * 128;
      int r = e / BK, kk = e % BK;
      int gr = bm + r, gk = k0 + kk;
      bool ok = gr < rows && gk < kpad;
      const cd* src = ok ? Q + (size_t)gr * ld + gk : Q;
      cp_async16(a + r * ASTR + kk, src, ok);
    }
#pragma unroll
    for (int it = 0; it < (BK * BN) / 128; ++it) {
      int e = tid + it * 128;
      int kk = e / BN, c = e % BN;
      int gk = k0 + kk, gc = bn + c;
      bool ok = gk < kpad && gc < ld;
      const cd* src = ok ? V + (size_t)gk * ld + gc : V;
      cp_async16(b + kk * BSTR + c, src, ok);
    }
  };

  double cr[2][4][4], ci[2][4][4];
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) cr[mi][ni][e] = ci[mi][ni][e] = 0.0;

  const int nk = kpad / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load_stage(s, s * BK);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    int nxt = kt + STAGES - 1;
    if (nxt < nk) load_stage(nxt % STAGES, nxt * BK);
    cp_async_commit();
    const cd* a = As + (kt % STAGES) * A_TILE;
    const cd* b = Bs + (kt % STAGES) * B_TILE;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      cd af[2][2], bf[4];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        af[mi][0] = a[(wm + mi * 16 + g) * ASTR + kk + t];
        af[mi][1] = a[(wm + mi * 16 + g + 8) * ASTR + kk + t];
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) bf[ni] = b[(kk + t) * BSTR + wn + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
          double* R = cr[mi][ni];
          double* I = ci[mi][ni];
          dmma(R[0], R[1], R[2], R[3], af[mi][0].x, af[mi][1].x, bf[ni].x);
          dmma(R[0], R[1], R[2], R[3], -af[mi][0].y, -af[mi][1].y, bf[ni].y);
          dmma(I[0], I[1], I[2], I[3], af[mi][0].x, af[mi][1].x, bf[ni].y);
          dmma(I[0], I[1], I[2], I[3], af[mi][0].y, af[mi][1].y, bf[ni].x);
        }
    }
  }
  cp_async_wait<0>();

  // fused epilogue: P += cb*(acc + Q o D_a); Qo = Q + ca*P
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        int r = bm + wm + mi * 16 + g + ((e >= 2) ? 8 : 0);
        int c = bn + wn + ni * 8 + 2 * t + (e & 1);
        if (r < rows && c < n) {
          int ang = r / n;
          size_t o = (size_t)r * ld + c;
          cd q = Q[o];
          cd d = D[(size_t)ang * ld + c];
          cd acc = cd{cr[mi][ni][e], ci[mi][ni][e]} + q * d;
          cd p = P[o] + cb * acc;
          P[o] = p;
          Qo[o] = q + ca * p;
        }
      }
  __syncthreads();  // the next tile's loads reuse the shared-memory stages
  }
}

void launch_stage_gemm_f64(const cd* Q, cd* P, cd* Qo, const cd* V, const cd* D, int nang, int n,
                           int ld, int kpad, double cb, double ca, cudaStream_t st,
                           StackedRows sr, int max_sms) {
  using namespace f64gemm;
  static SmemOptIn attr;
  attr.ensure((const void*)k_stage_gemm_f64, SMEM);
  int rows = nang * n;
  if (sr.rows_b <= 0) sr = StackedRows{rows, 0};
  const int nprob = ceil_div(rows, sr.rows_b);
  const int tiles_x = ceil_div(n, BN), tiles_y = nprob * ceil_div(sr.rows_b, BM);
  const int ntiles = tiles_x * tiles_y;
  if (max_sms > 0 && ntiles > 2 * max_sms) {  // two blocks per SM
    k_stage_gemm_f64<<<2 * max_sms, 128, SMEM, st>>>(Q, P, Qo, V, D, rows, n, ld, kpad, cb, ca, sr,
                                                     tiles_x, ntiles);
  } else {
    dim3 grid(tiles_x, tiles_y);
    k_stage_gemm_f64<<<grid, 128, SMEM, st>>>(Q, P, Qo, V, D, rows, n, ld, kpad, cb, ca, sr,
                                              tiles_x, ntiles);
  }
}

// ============================================================ identity / flags
__global__ void k_set_identity(cd* __restrict__ Q, const int* __restrict__ flag, int n, int ld) {
  int j = blockIdx.y * blockDim.x + threadIdx.x;
  int r = blockIdx.x;
  int a = r / n, i = r - a * n;
  if (j >= n) return;
  if (flag && !flag[a]) return;
  Q[(size_t)r * ld + j] = cd{i == j ? 1.0 : 0.0, 0.0};
}

void launch_set_identity(cd* Q, const int* flag, int nang, int n, int ld, cudaStream_t st) {
  dim3 grid(nang * n, ceil_div(n, 128));  // rows on x: more than 65535 stacked rows
  k_set_identity<<<grid, 128, 0, st>>>(Q, flag, n, ld);
}

// ============================================================ K7 Gershgorin estimate
__global__ void k_cond_est(const cd* __restrict__ Q, int n, int ld, int force,
                           int* __restrict__ flag, double* __restrict__ dval) {
  const int a = blockIdx.x;
  const cd* A = Q + (size_t)a * n * ld;
  double mn = INFINITY, mx = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double tsum = 0.0;
    for (int i = 0; i < n; ++i) {
      if (i != j) {
        cd v = A[(size_t)i * ld + j];
        tsum = tsum + sqrt(v.x * v.x + v.y * v.y);
      }
    }
    cd dj = A[(size_t)j * ld + j];
    double ad = hypot(dj.x, dj.y);
    mn = fmin(mn, ad - tsum);
    mx = fmax(mx, ad + tsum);
  }
  __shared__ double smn[32], smx[32];
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    smn[w] = mn;
    smx[w] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nw = (blockDim.x + 31) >> 5;
    for (int i = 1; i < nw; ++i) {
      mn = fmin(mn, smn[i]);
      mx = fmax(mx, smx[i]);
    }
    cd a11 = A[0];
    mx = fmax(mx, hypot(a11.x, a11.y));
    double d = (mn < 0.0) ? 1e100 : mx / mn;
    if (dval) dval[a] = d;
    flag[a] = (force || d > 1e3) ? 1 : 0;
  }
}

void launch_cond_est(const cd* Q, int nang, int n, int ld, int force, int* flag, double* dval,
                     cudaStream_t st) {
  k_cond_est<<<nang, 256, 0, st>>>(Q, n, ld, force, flag, dval);
}

// ============================================================ K8 blocked Gauss-Jordan
// [Q | P] -> [I | Q^{-1} P] with partial pivoting (pivot = max |re|+|im| among the
// rows not yet used, lowest index on ties, as zgetrf's izamax), in panels of
// kW = 16 columns.  Two implementations (launch_gauss_jordan picks by arithmetic
// and size):
// * shared memory (products-first arithmetic, and beyond 640 rows): the panel
//   kernel factors rows c0.. of the n x 16 panel in shared memory (LU with row
//   swaps) and forms W1 = B1^{-1} and the elimination multipliers L2 = B2 B1^{-1}
//   for every other row; the update kernel applies the swaps and
//     C1 <- W1 C1,   C2 <- C2 - L2 C1
//   to all remaining columns (Q columns right of the panel and every P column),
//   one thread per column.  (24-column panels, which fit shared memory up to
//   n = 530, measured slower at n = 521: the serial column steps outweigh the
//   saved passes over the trailing matrix.)
// * row per thread (the renormalisations, n <= 640): k_gj_panel_rows eliminates
//   the panel in place with each row in one thread's registers and writes E; the
//   trailing update C' = C + E C1 runs on the FP64 tensor path
//   (k_gj_update_mma), rank 32 in the split forms.
constexpr int kWMax = 16;      // panel width the scratch is sized for
constexpr int kUpdCols = 128;  // trailing columns per update block

struct GJScratch {
  int* piv;   // nang x 2 kW
  cd* W1;     // nang x kW x kW
  cd* L2;     // nang x n x 2 kW (the shared-memory path uses nang x n x kW of it)
};

// Pivots and multipliers: 2 kW per angle (the row-per-thread path keeps the pivots
// and E of two panels; the shared-memory path uses the first kW of each).
size_t gj_scratch_bytes(int nang, int n) {
  size_t b = (size_t)nang * 2 * kWMax * sizeof(int);
  b = (b + 255) & ~size_t(255);
  b += (size_t)nang * kWMax * kWMax * sizeof(cd);
  b = (b + 255) & ~size_t(255);
  b += (size_t)nang * n * 2 * kWMax * sizeof(cd);
  return b + 256;
}

static GJScratch gj_carve(void* scratch, int nang, int n) {
  GJScratch s;
  char* p = reinterpret_cast<char*>(scratch);
  s.piv = reinterpret_cast<int*>(p);
  size_t b = (size_t)nang * 2 * kWMax * sizeof(int);
  b = (b + 255) & ~size_t(255);
  s.W1 = reinterpret_cast<cd*>(p + b);
  b += (size_t)nang * kWMax * kWMax * sizeof(cd);
  b = (b + 255) & ~size_t(255);
  s.L2 = reinterpret_cast<cd*>(p + b);
  return s;
}

// Complex multiply-add of the elimination: kF selects four fused multiply-adds
// (the split forms' renormalisations) or the product formed first (the FP64
// form, whose results match the reference's rounding most closely).
template <bool kF>
__device__ __forceinline__ cd gj_add(cd s, cd a, cd b) {
  if constexpr (kF) return cfma(a, b, s);
  else return s + a * b;
}
template <bool kF>
__device__ __forceinline__ cd gj_sub(cd s, cd a, cd b) {
  if constexpr (kF) return cfms(a, b, s);
  else return s - a * b;
}

// Column-major complex access helper for the panel held in shared memory: S[i*kW + k].
template <int kW, bool kF>
__global__ void k_gj_panel(const cd* __restrict__ Q, const int* __restrict__ flag, int n, int ld,
                           int c0, int w, GJScratch sc, unsigned* status) {
  const int a = blockIdx.x;
  if (flag && !flag[a]) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* S = reinterpret_cast<cd*>(smem_raw);  // n x kW
  __shared__ double rv[32];
  __shared__ int ri[32];
  __shared__ int s_piv;
  __shared__ cd Linv[kW * kW], Uinv[kW * kW], W1s[kW * kW];
  const cd* A = Q + (size_t)a * n * ld;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * kW; e += nt) {
    int i = e / kW, k = e % kW;
    S[e] = (k < w) ? A[(size_t)i * ld + c0 + k] : cd{0.0, 0.0};
  }
  __syncthreads();
  // ---- LU with partial pivoting of rows c0..n-1 of the panel
  for (int jj = 0; jj < w; ++jj) {
    const int col = c0 + jj;
    double best = -1.0;
    int bi = n;
    for (int i = col + tid; i < n; i += nt) {
      double v = cabs1(S[i * kW + jj]);
      if (v > best) {  // strict: keeps the lowest index within this thread's strided scan
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if ((tid & 31) == 0) {
      rv[tid >> 5] = best;
      ri[tid >> 5] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      int nw = (nt + 31) >> 5;
      for (int q = 1; q < nw; ++q)
        if (rv[q] > best || (rv[q] == best && ri[q] < bi)) {
          best = rv[q];
          bi = ri[q];
        }
      if (bi >= n) bi = col;
      s_piv = bi;
      sc.piv[a * kW + jj] = bi;
    }
    __syncthreads();
    const int p = s_piv;
    if (p != col) {
      for (int k = tid; k < kW; k += nt) {
        cd tmp = S[col * kW + k];
        S[col * kW + k] = S[p * kW + k];
        S[p * kW + k] = tmp;
      }
    }
    __syncthreads();
    const cd d = S[col * kW + jj];
    if (d.x == 0.0 && d.y == 0.0) {
      if (tid == 0) atomicOr(status, kStatusZeroPivot);
    }
    const cd rinv = cdiv(cd{1.0, 0.0}, d);
    for (int i = col + 1 + tid; i < n; i += nt) {
      cd l = S[i * kW + jj] * rinv;
      S[i * kW + jj] = l;
      for (int k = jj + 1; k < w; ++k) S[i * kW + k] = gj_sub<kF>(S[i * kW + k], l, S[col * kW + k]);
    }
    __syncthreads();
  }
  // ---- inverses of the unit-lower L11 and upper U11 (w x w), W1 = U11^{-1} L11^{-1}
  if (tid < kW) {
    const int k = tid;  // column k of each inverse
    for (int i = 0; i < kW; ++i) {  // forward substitution L11 x = e_k
      cd s = cd{(i == k) ? 1.0 : 0.0, 0.0};
      if (i < w)
        for (int m = 0; m < i; ++m) s = s - S[(c0 + i) * kW + m] * Linv[m * kW + k];
      Linv[i * kW + k] = (i < w && k < w) ? s : cd{0.0, 0.0};
    }
    for (int i = kW - 1; i >= 0; --i) {  // back substitution U11 x = e_k
      cd s = cd{(i == k) ? 1.0 : 0.0, 0.0};
      if (i < w && k < w) {
        for (int m = i + 1; m < w; ++m) s = s - S[(c0 + i) * kW + m] * Uinv[m * kW + k];
        s = cdiv(s, S[(c0 + i) * kW + i]);
      } else {
        s = cd{0.0, 0.0};
      }
      Uinv[i * kW + k] = s;
    }
  }
  __syncthreads();
  for (int e = tid; e < kW * kW; e += nt) {
    int i = e / kW, k = e % kW;
    cd s = cd{0.0, 0.0};
    for (int m = 0; m < kW; ++m) s = s + Uinv[i * kW + m] * Linv[m * kW + k];
    W1s[e] = s;
    sc.W1[(size_t)a * kW * kW + e] = s;
  }
  __syncthreads();
  // ---- multipliers: rows >= c0+w: L21 L11^{-1};  rows < c0: B0 W1
  cd* L2 = sc.L2 + (size_t)a * n * kW;
  for (int e = tid; e < n * kW; e += nt) {
    int i = e / kW, k = e % kW;
    cd s = cd{0.0, 0.0};
    if (k < w) {
      if (i >= c0 + w) {
        for (int m = 0; m < w; ++m) s = gj_add<kF>(s, S[i * kW + m], Linv[m * kW + k]);
      } else if (i < c0) {
        for (int m = 0; m < w; ++m) s = gj_add<kF>(s, S[i * kW + m], W1s[m * kW + k]);
      }
    }
    L2[e] = s;
  }
}

// Panel step for n <= kPanelRowsMax rows, one row per thread: Gauss-Jordan
// elimination of the panel columns in place, with the pivot rule of k_gj_panel.
// Column step jj pivots, swaps rows col and p, scales the pivot row by r = 1/d and
// eliminates the column from every other row i with the multiplier g = f_i r
// (f_i the row's entry in column jj): x_k <- x_k - g u_k for the other columns,
// and the freed slot jj takes -g.  After w steps the panel holds E with
// E [B1; B_other] = [I; 0] over the pivot columns: its pivot rows are B1^{-1}, its
// other rows -B_other B1^{-1}.  The trailing update is then, after the same row
// swaps, C1' = E_pivot C1 for the pivot rows and C' = C + E_i C1 for the others.
// One barrier per column: each warp publishes its best candidate row, and the
// owner of row col publishes that row, before it.
constexpr int kPanelRowsMax = 640;
template <bool kF, int kMaxT>
__global__ void __launch_bounds__(kMaxT, 1)
    k_gj_panel_rows(const cd* __restrict__ Q, const int* __restrict__ flag, int n, int ld, int c0,
                    int w, int* __restrict__ piv, int pstride, cd* __restrict__ E, int estride,
                    unsigned* status) {
  static_assert(kWMax == 16, "one 16-column panel per thread row");
  const int a = blockIdx.x;
  if (flag && !flag[a]) return;
  constexpr int kMaxWarps = kMaxT / 32;
  __shared__ double cand_v[2][kMaxWarps];
  __shared__ int cand_i[2][kMaxWarps];
  __shared__ cd cand_row[2][kMaxWarps][kWMax];
  __shared__ cd crow[2][kWMax];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
  const unsigned full = 0xffffffffu;
  cd x[kWMax];
  {
    const cd* A = Q + (size_t)a * n * ld + (size_t)min(tid, n - 1) * ld + c0;
#pragma unroll
    for (int k = 0; k < kWMax; ++k) x[k] = (tid < n && k < w) ? A[k] : cd{0.0, 0.0};
  }
  // a runtime loop over the columns (an unrolled one overflows the instruction
  // cache); column jj of the row is picked by a select over the 16 registers
  for (int jj = 0; jj < w; ++jj) {
    const int col = c0 + jj, buf = jj & 1;
    // ---- this warp's candidate: max |re|+|im| over rows >= col, lowest row on ties
    cd xj = x[0];
#pragma unroll
    for (int k = 1; k < kWMax; ++k)
      if (k == jj) xj = x[k];
    const bool live = tid >= col && tid < n;
    double best = live ? cabs1(xj) : -1.0;
    int bi = live ? tid : n;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(full, best, o);
      const int oi = __shfl_xor_sync(full, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (tid == bi) {
#pragma unroll
      for (int k = 0; k < kWMax; ++k) cand_row[buf][warp][k] = x[k];
    }
    if (lane == 0) {
      cand_v[buf][warp] = best;
      cand_i[buf][warp] = bi;
    }
    if (tid == col) {
#pragma unroll
      for (int k = 0; k < kWMax; ++k) crow[buf][k] = x[k];
    }
    __syncthreads();
    // ---- the block's pivot among the warp candidates
    best = (lane < nw) ? cand_v[buf][lane] : -1.0;
    bi = (lane < nw) ? cand_i[buf][lane] : n;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(full, best, o);
      const int oi = __shfl_xor_sync(full, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    const int p = __shfl_sync(full, bi, 0), pw = p >> 5;  // row p is thread p's
    if (tid == 0) piv[a * pstride + jj] = p;
    const cd* u = cand_row[buf][pw];  // the pivot row (old row p)
    const cd d = u[jj];  // shared memory: a dynamic index is fine
    if (d.x == 0.0 && d.y == 0.0 && tid == 0) atomicOr(status, kStatusZeroPivot);
    const double dinv = 1.0 / (d.x * d.x + d.y * d.y);  // 1/d = conj(d) / |d|^2
    const cd r = cd{d.x * dinv, -d.y * dinv};
    if (tid == col) {
#pragma unroll
      for (int k = 0; k < kWMax; ++k) x[k] = (k == jj) ? r : u[k] * r;
    } else {
      if (tid == p) {  // row p now holds the old row col
#pragma unroll
        for (int k = 0; k < kWMax; ++k) x[k] = crow[buf][k];
        xj = crow[buf][jj];
      }
      const cd g = xj * r;
#pragma unroll
      for (int k = 0; k < kWMax; ++k) x[k] = (k == jj) ? -g : gj_sub<kF>(x[k], g, u[k]);
    }
  }
  if (tid < n) {
    cd* e = E + ((size_t)a * n + tid) * estride;
#pragma unroll
    for (int k = 0; k < kWMax; ++k) e[k] = x[k];
  }
}

// Each CTA owns kUpdCols of the remaining columns of one angle.
// One thread per column of the trailing matrix (Q columns right of the panel,
// then every P column), 128 columns per block: the column's pivot-row values C1
// stay in registers; the multipliers L2 of 32 rows at a time are copied into
// shared memory asynchronously (two buffers: the next chunk is in flight while the
// current one is applied) and read as broadcasts.  At most 128 registers per
// thread, so four blocks share an SM and the 9 column blocks of all 61 angles of
// an N = 521 solve run in one wave.
constexpr int kUpdRows = 32;
template <int kW, bool kF>
__global__ void __launch_bounds__(kUpdCols, 4) k_gj_update(cd* __restrict__ Q, cd* __restrict__ P,
                                                           const int* __restrict__ flag, int n,
                                                           int ld, int c0, int w, GJScratch sc) {
  const int a = blockIdx.y;
  if (flag && !flag[a]) return;
  const int qrest = n - (c0 + w);          // Q columns right of the panel
  const int vc = blockIdx.x * kUpdCols + threadIdx.x;  // virtual column
  const int total = qrest + n;
  __shared__ cd W1[kW * kW];
  __shared__ __align__(16) cd Ls[2][kUpdRows][kW];  // 16-byte cp.async targets
  __shared__ int piv[kW];
  const int tid = threadIdx.x;
  for (int e = tid; e < kW * kW; e += kUpdCols) W1[e] = sc.W1[(size_t)a * kW * kW + e];
  if (tid < kW) piv[tid] = sc.piv[a * kW + tid];
  const cd* L2 = sc.L2 + (size_t)a * n * kW;
  constexpr int kStage = kUpdRows * kW / kUpdCols;  // multiplier entries per thread and chunk
  static_assert(kUpdRows * kW % kUpdCols == 0, "chunk staging");
  // asynchronous copies of the chunk at rows i0.. into Ls[b] (zeros past row n)
  auto fetch = [&](int i0, int b) {
#pragma unroll
    for (int q = 0; q < kStage; ++q) {
      const int e = tid + q * kUpdCols, i = i0 + e / kW;
      const cd* src = L2 + (size_t)min(i, n - 1) * kW + e % kW;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&Ls[b][e / kW][e % kW]);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                   "r"(i < n ? 16 : 0)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  fetch(0, 0);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  const bool valid = vc < total;
  cd* base = nullptr;
  if (valid) base = (vc < qrest) ? Q + (size_t)a * n * ld + (c0 + w + vc)
                                 : P + (size_t)a * n * ld + (vc - qrest);
  // row swaps in order, then C1 = the pivot rows (values after the swaps)
  cd c1[kW];
  if (valid) {
    for (int jj = 0; jj < w; ++jj) {
      const int r0 = c0 + jj, r1 = piv[jj];
      if (r1 != r0) {
        const cd t0 = base[(size_t)r0 * ld], t1 = base[(size_t)r1 * ld];
        base[(size_t)r0 * ld] = t1;
        base[(size_t)r1 * ld] = t0;
      }
    }
#pragma unroll
    for (int k = 0; k < kW; ++k) c1[k] = (k < w) ? base[(size_t)(c0 + k) * ld] : cd{0.0, 0.0};
    // pivot rows <- W1 C1
    for (int k = 0; k < w; ++k) {
      cd v = cd{0.0, 0.0};
#pragma unroll
      for (int m = 0; m < kW; ++m)
        if (m < w) v = gj_add<kF>(v, W1[k * kW + m], c1[m]);  // entries past w are not written
      base[(size_t)(c0 + k) * ld] = v;
    }
  }
  // other rows <- C2 - L2 C1
  int buf = 0;
  for (int i0 = 0; i0 < n; i0 += kUpdRows, buf ^= 1) {
    if (i0 + kUpdRows < n) fetch(i0 + kUpdRows, buf ^ 1);
    if (valid) {
      constexpr int U = 8;
      for (int q = 0; q < kUpdRows; q += U) {
        cd v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int i = i0 + q + u;
          const bool row = i < n && !(i >= c0 && i < c0 + w);
          v[u] = row ? base[(size_t)i * ld] : cd{0.0, 0.0};
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int i = i0 + q + u;
          if (i < n && !(i >= c0 && i < c0 + w)) {
            cd x = v[u];
#pragma unroll
            for (int m = 0; m < kW; ++m)
              if (m < w) x = gj_sub<kF>(x, Ls[buf][q + u][m], c1[m]);
            base[(size_t)i * ld] = x;
          }
        }
      }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }
}

// Trailing update from a Gauss-Jordan step's E on the FP64 tensor path (fused
// rounding).  For the kW pivot rows c0..c0+w-1 (w <= kW) the step is, after its
// row swaps, C' = C + E C1 for every row (C = 0 for the pivot rows, whose E rows
// are B1^{-1}): a complex GEMM with K = kW over the trailing columns.  The columns
// come in two segments (Q right of the panel and P; or the 16 columns of another
// step's E), each with its own base, row stride and angle stride.  The CTA owns
// kMmaCols columns of one angle; after a common setup its four warps work
// independently on 16-row strips (warp w: strips w, w+4, ...).  Per strip: m16n8k4
// FP64 MMAs, four real MMAs per complex product, accumulators initialised from C;
// the warp's E rows come through its own two cp.async buffers and the next strip's
// C values are loaded into registers while the current strip's MMAs run.
// Row swaps: warp 0 replays the step's swap sequence on the (at most 2 kW) touched
// row positions, so every position knows which original row its value comes from;
// C1 (the pivot rows after the swaps) and the values that end in touched rows
// below the pivot block are read into shared memory before any row is written,
// and a strip reads a touched row from that stash.
constexpr int kMmaCols = 32;        // complex columns per CTA (4 n8 tiles)
constexpr int kStrip = 16;          // rows per warp strip
constexpr int kC1Str = kMmaCols + 2;
template <int kW>
struct MmaUpdSmem {
  static constexpr int kEStr = kW + 4;  // complex entries per E row in shared memory
  cd E[4][2][kStrip][kEStr];
  cd C1[kW][kC1Str];
  cd stash[kW][kMmaCols];
  short rslot[kMaxBeams];
  int tpos[2 * kW], tsrc[2 * kW];
  int ntouched;
};

// Trailing columns of an update: segment 0 (n0 columns) then segment 1.  Element
// (r, vc) of angle a is p + a * as + r * ld + vc (vc counted within its segment).
struct GjCols {
  cd* p0;
  long long as0;
  int ld0, n0;
  cd* p1;
  long long as1;
  int ld1, n1;
};

// One work item: angle a, trailing columns vc0 .. vc0 + kMmaCols - 1.
template <int kW>
__device__ __forceinline__ void gj_update_mma_item(MmaUpdSmem<kW>& sm, const GjCols& cols, int n,
                                                   int c0, int w, const int* __restrict__ pivs,
                                                   int pstride, const cd* __restrict__ E,
                                                   int estride, int a, int vc0) {
  constexpr int kNi = kMmaCols / 8, kSlots = (2 * kW + 31) / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int total = cols.n0 + cols.n1;
  cd* const b0 = cols.p0 + (size_t)a * cols.as0;
  cd* const b1 = cols.p1 + (size_t)a * cols.as1;
  // element (r, vc) of this angle's trailing columns (vc < total)
  auto at = [&](int r, int vc) -> cd* {
    return vc < cols.n0 ? b0 + (size_t)r * cols.ld0 + vc
                        : b1 + (size_t)r * cols.ld1 + (vc - cols.n0);
  };
  const cd* Ea = E + (size_t)a * n * estride;
  const int* pa = pivs + (size_t)a * pstride;
  for (int i = tid; i < n; i += 128) sm.rslot[i] = -1;
  __syncthreads();
  if (warp == 0) {
    // entry q (lane q & 31, slot q >> 5) holds a touched position and the row its
    // value comes from: entries 0..w-1 are the pivot block, later ones the pivot
    // rows below it in order of first use
    int pos[kSlots], src[kSlots], myp[kSlots];
#pragma unroll
    for (int e = 0; e < kSlots; ++e) {
      const int q = lane + 32 * e;
      pos[e] = q < w ? c0 + q : -1;
      src[e] = pos[e];
      myp[e] = q < w ? pa[q] : 0;
    }
    int nt = w;
    for (int jj = 0; jj < w; ++jj) {
      int r1 = 0;
#pragma unroll
      for (int e = 0; e < kSlots; ++e)
        if ((jj >> 5) == e) r1 = __shfl_sync(0xffffffffu, myp[e], jj & 31);
      int i1 = -1;
#pragma unroll
      for (int e = kSlots - 1; e >= 0; --e) {
        const unsigned hit = __ballot_sync(0xffffffffu, pos[e] == r1);
        if (hit) i1 = 32 * e + __ffs(hit) - 1;
      }
      if (i1 < 0) {
        i1 = nt++;
#pragma unroll
        for (int e = 0; e < kSlots; ++e)
          if (lane + 32 * e == i1) pos[e] = src[e] = r1;
      }
      int sj = 0, si = 0;
#pragma unroll
      for (int e = 0; e < kSlots; ++e) {
        const int vj = __shfl_sync(0xffffffffu, src[e], jj & 31);
        const int vi = __shfl_sync(0xffffffffu, src[e], i1 & 31);
        if ((jj >> 5) == e) sj = vj;
        if ((i1 >> 5) == e) si = vi;
      }
#pragma unroll
      for (int e = 0; e < kSlots; ++e) {
        if (lane + 32 * e == jj) src[e] = si;
        if (lane + 32 * e == i1) src[e] = sj;
      }
    }
#pragma unroll
    for (int e = 0; e < kSlots; ++e) {
      const int q = lane + 32 * e;
      if (q < 2 * kW) {
        sm.tpos[q] = pos[e];
        sm.tsrc[q] = src[e];
      }
      if (q >= w && q < nt) sm.rslot[pos[e]] = (short)(q - w);
    }
    if (lane == 0) sm.ntouched = nt;
  }
  __syncthreads();
  {
    const int nt = sm.ntouched;
#pragma unroll
    for (int it = 0; it < 2 * kW * kMmaCols / 128; ++it) {
      const int e = tid + it * 128, q = e / kMmaCols, c = e % kMmaCols, vc = vc0 + c;
      if (q < kW) {
        sm.C1[q][c] = (q < w && vc < total) ? *at(sm.tsrc[q], vc) : cd{0.0, 0.0};
      } else {  // stash slot sl: touched entry w + sl (rows below the pivot block)
        const int sl = q - kW, te = w + sl;
        if (te < nt) sm.stash[sl][c] = vc < total ? *at(sm.tsrc[te], vc) : cd{0.0, 0.0};
      }
    }
  }
  __syncthreads();
  // this thread's 8 columns are vc0 + ni * 8 + 2t + j; addresses formed on use
  const int vt = vc0 + 2 * t;
  auto fetch_e = [&](int strip, int b) {
#pragma unroll
    for (int q = 0; q < kStrip * kW / 32; ++q) {
      const int e = lane + q * 32, r = e / kW, k = e % kW, row = strip * kStrip + r;
      const cd* src = Ea + (size_t)min(row, n - 1) * estride + k;
      const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sm.E[warp][b][r][k]);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                   "r"(row < n ? 16 : 0)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // C values of a strip in accumulator order (0 in the pivot rows, stash values in
  // touched rows)
  auto load_c = [&](int strip, double (&cr)[kNi][4], double (&ci)[kNi][4]) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = strip * kStrip + g + 8 * h;
      const bool live = r < n && !(r >= c0 && r < c0 + w);
      const int sl = live ? sm.rslot[r] : -1;
#pragma unroll
      for (int ni = 0; ni < kNi; ++ni)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int vc = vt + ni * 8 + j;
          cd v = cd{0.0, 0.0};
          if (live && vc < total) v = sl >= 0 ? sm.stash[sl][ni * 8 + 2 * t + j] : *at(r, vc);
          cr[ni][2 * h + j] = v.x;
          ci[ni][2 * h + j] = v.y;
        }
    }
  };
  const int nstrips = ceil_div(n, kStrip);
  double cr[kNi][4], ci[kNi][4];
  if (warp < nstrips) {
    fetch_e(warp, 0);
    load_c(warp, cr, ci);
  }
  int b = 0;
  for (int strip = warp; strip < nstrips; strip += 4, b ^= 1) {
    const int nxt = strip + 4;
    double nr[kNi][4], nim[kNi][4];
    if (nxt < nstrips) {
      fetch_e(nxt, b ^ 1);
      load_c(nxt, nr, nim);
      asm volatile("cp.async.wait_group 1;" ::: "memory");
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncwarp();
#pragma unroll
    for (int kk = 0; kk < kW / 4; ++kk) {
      const cd a0 = sm.E[warp][b][g][kk * 4 + t];
      const cd a1 = sm.E[warp][b][g + 8][kk * 4 + t];
#pragma unroll
      for (int ni = 0; ni < kNi; ++ni) {
        const cd bf = sm.C1[kk * 4 + t][ni * 8 + g];
        double* R = cr[ni];
        double* I = ci[ni];
        dmma(R[0], R[1], R[2], R[3], a0.x, a1.x, bf.x);
        dmma(R[0], R[1], R[2], R[3], -a0.y, -a1.y, bf.y);
        dmma(I[0], I[1], I[2], I[3], a0.x, a1.x, bf.y);
        dmma(I[0], I[1], I[2], I[3], a0.y, a1.y, bf.x);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = strip * kStrip + g + 8 * h;
      if (r < n) {
#pragma unroll
        for (int ni = 0; ni < kNi; ++ni)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int vc = vt + ni * 8 + j;
            if (vc < total) *at(r, vc) = cd{cr[ni][2 * h + j], ci[ni][2 * h + j]};
          }
      }
    }
    __syncwarp();  // the next fetch reuses this strip's buffer
    if (nxt < nstrips) {
#pragma unroll
      for (int ni = 0; ni < kNi; ++ni)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          cr[ni][e] = nr[ni][e];
          ci[ni][e] = nim[ni][e];
        }
    }
  }
}

// Grid-stride over the (angle, column tile) items, so the last wave of a launch is
// not left partly empty.
template <int kW>
__global__ void __launch_bounds__(128, kW == 16 ? 3 : 2)
    k_gj_update_mma(GjCols cols, const int* __restrict__ flag, int n, int c0, int w,
                    const int* __restrict__ pivs, int pstride, const cd* __restrict__ E,
                    int estride, int nang) {
  extern __shared__ __align__(16) unsigned char mma_dyn[];
  MmaUpdSmem<kW>& sm = *reinterpret_cast<MmaUpdSmem<kW>*>(mma_dyn);
  const int tiles = ceil_div(cols.n0 + cols.n1, kMmaCols);
  for (int item = blockIdx.x; item < tiles * nang; item += gridDim.x) {
    const int a = item / tiles;
    if (flag && !flag[a]) continue;
    gj_update_mma_item<kW>(sm, cols, n, c0, w, pivs, pstride, E, estride, a,
                           (item - a * tiles) * kMmaCols);
    __syncthreads();  // the next item reuses the shared memory
  }
}

// The original path: the shared-memory panel (W1, L2 by triangular inverses) and
// the one-thread-per-column update, for the product-first arithmetic (the boundary
// transforms, the bulk solve) and for more than kPanelRowsMax rows.
template <int kW, bool kF>
static void gauss_jordan_smem(cd* Q, cd* P, const int* flag, int nang, int n, int ld,
                              const GJScratch& sc, unsigned* status, cudaStream_t st) {
  static SmemOptIn attr;
  const size_t smem = (size_t)n * kW * sizeof(cd);
  attr.ensure((const void*)k_gj_panel<kW, kF>, smem);
  for (int c0 = 0; c0 < n; c0 += kW) {
    const int w = (n - c0 < kW) ? n - c0 : kW;
    k_gj_panel<kW, kF><<<nang, 256, smem, st>>>(Q, flag, n, ld, c0, w, sc, status);
    const int total = (n - (c0 + w)) + n;
    dim3 grid(ceil_div(total, kUpdCols), nang);
    k_gj_update<kW, kF><<<grid, kUpdCols, 0, st>>>(Q, P, flag, n, ld, c0, w, sc);
  }
}

static int gj_sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

// The renormalisations, n <= 640: the row-per-thread panel (fused or product-first
// complex arithmetic) and the trailing update on the FP64 tensor path.  The split
// forms take 32 pivot columns per trailing update.  For columns c0..c0+31: the panel on the first 16
// (E_a), a rank-16 update of the next 16 columns only, the panel on those (E_b),
// the second step applied to E_a's 16 columns (so that [E_a | E_b] is the E of a
// 32-column Gauss-Jordan step: the in-place elimination of the second half would
// have updated the first half's slots), then one rank-32 update of every other
// trailing column with the 32 row swaps in order.  The last panel of fewer than
// 17 columns takes one rank-16 step.  E and the pivots live in the scratch's
// 32-column blocks (row stride 32).
template <bool kF>
static void gauss_jordan_rows(cd* Q, cd* P, const int* flag, int nang, int n, int ld,
                              const GJScratch& sc, unsigned* status, cudaStream_t st) {
  static SmemOptIn attr16, attr32;
  attr16.ensure((const void*)k_gj_update_mma<16>, sizeof(MmaUpdSmem<16>));
  attr32.ensure((const void*)k_gj_update_mma<32>, sizeof(MmaUpdSmem<32>));
  const int threads = round_up(n, 32), sms = gj_sm_count();
  constexpr int kP = 2 * kWMax;  // pivots and E columns per angle in the scratch
  const long long qa = (long long)n * ld, ea = (long long)n * kP;
  auto panel = [&](int c, int w, int poff) {
    int* pv = sc.piv + poff;
    cd* E = sc.L2 + poff;
    if (threads <= 256)
      k_gj_panel_rows<kF, 256><<<nang, threads, 0, st>>>(Q, flag, n, ld, c, w, pv, kP, E, kP,
                                                         status);
    else if (threads <= 544)
      k_gj_panel_rows<kF, 544><<<nang, threads, 0, st>>>(Q, flag, n, ld, c, w, pv, kP, E, kP,
                                                         status);
    else
      k_gj_panel_rows<kF, kPanelRowsMax><<<nang, threads, 0, st>>>(Q, flag, n, ld, c, w, pv, kP,
                                                                   E, kP, status);
  };
  auto update16 = [&](const GjCols& cols, int c, int w, int poff) {
    const int items = ceil_div(cols.n0 + cols.n1, kMmaCols) * nang;
    if (items == 0) return;
    k_gj_update_mma<16><<<std::min(items, 3 * sms), 128, sizeof(MmaUpdSmem<16>), st>>>(
        cols, flag, n, c, w, sc.piv + poff, kP, sc.L2 + poff, kP, nang);
  };
  if (!kF) {
    // the FP64 form: rank-16 steps throughout (its parity against the reference's
    // test521 sp6 0.68 output, 2e-9, holds with this blocking and not with the
    // rank-32 one, 2.5e-9)
    for (int c0 = 0; c0 < n; c0 += kWMax) {
      const int w = std::min(kWMax, n - c0);
      panel(c0, w, 0);
      update16(GjCols{Q + c0 + w, qa, ld, n - c0 - w, P, qa, ld, n}, c0, w, 0);
    }
    return;
  }
  for (int c0 = 0; c0 < n;) {
    const int rem = n - c0;
    if (rem <= kWMax) {  // one rank-16 step: Q right of the panel (none) and P
      panel(c0, rem, 0);
      update16(GjCols{Q + c0 + rem, qa, ld, 0, P, qa, ld, n}, c0, rem, 0);
      break;
    }
    const int wb = std::min(kWMax, rem - kWMax), w = kWMax + wb;
    panel(c0, kWMax, 0);
    // step a on the next panel's columns only
    update16(GjCols{Q + c0 + kWMax, qa, ld, wb, P, qa, ld, 0}, c0, kWMax, 0);
    panel(c0 + kWMax, wb, kWMax);
    // step b on E_a's 16 columns
    update16(GjCols{sc.L2, ea, kP, kWMax, P, qa, ld, 0}, c0 + kWMax, wb, kWMax);
    // both steps on every other trailing column
    const GjCols rest{Q + c0 + w, qa, ld, n - c0 - w, P, qa, ld, n};
    const int items = ceil_div(rest.n0 + rest.n1, kMmaCols) * nang;
    k_gj_update_mma<32><<<std::min(items, 2 * sms), 128, sizeof(MmaUpdSmem<32>), st>>>(
        rest, flag, n, c0, w, sc.piv, kP, sc.L2, kP, nang);
    c0 += w;
  }
}

void launch_gauss_jordan(cd* Q, cd* P, const int* flag, int nang, int n, int ld, void* scratch,
                         unsigned* status, cudaStream_t st, int arith) {
  GJScratch sc = gj_carve(scratch, nang, n);
  const bool rows = n <= kPanelRowsMax;
  if (arith == kGjFused) {
    if (rows) gauss_jordan_rows<true>(Q, P, flag, nang, n, ld, sc, status, st);
    else gauss_jordan_smem<kWMax, true>(Q, P, flag, nang, n, ld, sc, status, st);
  } else if (arith == kGjFp64Mma && rows) {
    gauss_jordan_rows<false>(Q, P, flag, nang, n, ld, sc, status, st);
  } else {
    gauss_jordan_smem<kWMax, false>(Q, P, flag, nang, n, ld, sc, status, st);
  }
}

// ============================================================ RK4 stage combination
// After the product KP = A M of RK4 stage j (0..3, rk4_int surf_rk.f90:27-91):
// the stage derivative is k_j = (kq, KP) with kq = P (j = 0) or Pt; accumulate
// SQ/SP = k1 + 2 k2 + 2 k3 + k4 in that order, form the next stage point
// (Qt, Pt) = (Q, P) + step k_j, and after the last stage (Q, P) += dz/6 (SQ, SP).
// KP is cleared for the next product.  Only the n x n block is touched.
__global__ void k_rk4_combine(cd* __restrict__ Q, cd* __restrict__ P, cd* __restrict__ Qt,
                              cd* __restrict__ Pt, cd* __restrict__ KP, cd* __restrict__ SQ,
                              cd* __restrict__ SP, int j, double w, double step, double h6, int n,
                              int ld) {
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  const int r = blockIdx.x;
  if (c >= n) return;
  const size_t o = (size_t)r * ld + c;
  const cd kq = (j == 0) ? P[o] : Pt[o];
  const cd kp = KP[o];
  cd sq, sp;
  if (j == 0) {
    sq = kq;
    sp = kp;
  } else {
    sq = SQ[o] + w * kq;
    sp = SP[o] + w * kp;
  }
  if (j < 3) {
    SQ[o] = sq;
    SP[o] = sp;
    Qt[o] = Q[o] + step * kq;
    Pt[o] = P[o] + step * kp;
  } else {
    Q[o] = Q[o] + h6 * sq;
    P[o] = P[o] + h6 * sp;
  }
  KP[o] = cd{0.0, 0.0};
}

void launch_rk4_combine(cd* Q, cd* P, cd* Qt, cd* Pt, cd* KP, cd* SQ, cd* SP, int j, double w,
                        double step, double h6, int nang, int n, int ld, cudaStream_t st) {
  dim3 grid(nang * n, ceil_div(n, 128));  // rows on x: more than 65535 stacked rows
  k_rk4_combine<<<grid, 128, 0, st>>>(Q, P, Qt, Pt, KP, SQ, SP, j, w, step, h6, n, ld);
}

// ============================================================ boundary transforms
__global__ void k_invstransh_build(const cd* __restrict__ F, cd* __restrict__ Q,
                                   cd* __restrict__ P, int n, int ld) {
  int j = blockIdx.y * blockDim.x + threadIdx.x;
  int r = blockIdx.x;
  if (j >= n) return;
  int a = r / n, i = r - a * n;
  cd fh = conj(F[((size_t)a * n + j) * n + i]);  // F^H(i,j) = conj(F(j,i))
  size_t o = (size_t)r * ld + j;
  if (i == j) {
    Q[o] = cd{1.0 + fh.x, fh.y};
    P[o] = cd{1.0 - fh.x, -fh.y};
  } else {
    Q[o] = fh;
    P[o] = -fh;
  }
}

void launch_invstransh_build(const cd* F, cd* Q, cd* P, int nang, int n, int ld, cudaStream_t st) {
  dim3 grid(nang * n, ceil_div(n, 128));  // rows on x: more than 65535 stacked rows
  k_invstransh_build<<<grid, 128, 0, st>>>(F, Q, P, n, ld);
}

__global__ void k_invstransh_finish(cd* __restrict__ P, const cd* __restrict__ gam, int n,
                                    int ld) {
  int j = blockIdx.y * blockDim.x + threadIdx.x;
  int r = blockIdx.x;
  if (j >= n) return;
  int a = r / n, i = r - a * n;
  size_t o = (size_t)r * ld + j;
  P[o] = (cd{0.0, 1.0} * P[o]) * conj(gam[(size_t)a * n + i]);
}

void launch_invstransh_finish(cd* P, const cd* gam, int nang, int n, int ld, cudaStream_t st) {
  dim3 grid(nang * n, ceil_div(n, 128));  // rows on x: more than 65535 stacked rows
  k_invstransh_finish<<<grid, 128, 0, st>>>(P, gam, n, ld);
}

__global__ void k_stransh_build(cd* __restrict__ Q, cd* __restrict__ P, const cd* __restrict__ gam,
                                int n, int ld) {
  int j = blockIdx.y * blockDim.x + threadIdx.x;
  int r = blockIdx.x;
  if (j >= n) return;
  int a = r / n, i = r - a * n;
  size_t o = (size_t)r * ld + j;
  cd p = P[o];
  if (i == j) {
    cd g = conj(gam[(size_t)a * n + i]);
    Q[o] = g + cd{0.0, -1.0} * p;
    P[o] = g + cd{0.0, 1.0} * p;
  } else {
    Q[o] = cd{0.0, -1.0} * p;
    P[o] = cd{0.0, 1.0} * p;
  }
}

void launch_stransh_build(cd* Q, cd* P, const cd* gam, int nang, int n, int ld, cudaStream_t st) {
  dim3 grid(nang * n, ceil_div(n, 128));  // rows on x: more than 65535 stacked rows
  k_stransh_build<<<grid, 128, 0, st>>>(Q, P, gam, n, ld);
}

__global__ void k_intensities(const cd* __restrict__ R, const cd* __restrict__ gam,
                              const double* __restrict__ wnsga2, int n, int ld, int nb0,
                              double* __restrict__ f2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int a = blockIdx.y;
  if (i >= n) return;
  double s = gam[(size_t)a * n + i].x;
  double out = 0.0;
  if (s > 1e-10) {
    cd f = conj(R[((size_t)a * n + nb0) * ld + i]);  // f(i, nb0) = conj(R(nb0, i))
    out = (f * conj(f)).x * wnsga2[a] / s;
  }
  f2[(size_t)a * n + i] = out;
}

void launch_intensities(const cd* R, const cd* gam, const double* wnsga2, int nang, int n, int ld,
                        int nb0, double* f2, cudaStream_t st) {
  dim3 grid(ceil_div(n, 128), nang);
  k_intensities<<<grid, 128, 0, st>>>(R, gam, wnsga2, n, ld, nb0, f2);
}

__global__ void k_check_finite(const cd* __restrict__ X, size_t count, unsigned* status) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  for (; i < count; i += (size_t)gridDim.x * blockDim.x) {
    cd v = X[i];
    if (!isfinite(v.x) || !isfinite(v.y)) bad = true;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, kStatusNonFinite);
}

void launch_check_finite(const cd* X, size_t count, unsigned* status, cudaStream_t st) {
  k_check_finite<<<148 * 4, 256, 0, st>>>(X, count, status);
}

}  // namespace trhepd

namespace trhepd {

// ============================================================ rocking-curve convolution
// make_convolution.py (str-lapack/tool/make_convolution.py:21-29, 97-109): rows in
// blocks of `scan` consecutive angles; within a block
//   out[i][b] = sum_k f2[k][b] g(theta_i - theta_k) dtheta,  dtheta = theta_1 - theta_0,
//   g(x) = exp(-x^2 / (2 sigma^2)) / (sigma sqrt(2 pi)),     sigma = omega / (2 sqrt(2 ln 2)),
// summed in the script's order.  One thread per (row, beam).
__global__ void k_rocking_convolution(const double* __restrict__ ang,
                                      const double* __restrict__ f2, int rows, int scan, int nb,
                                      double sigma, double* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (b >= nb || i >= rows) return;
  const int b0 = (i / scan) * scan;
  const double d = ang[b0 + 1] - ang[b0];
  const double norm = 1.0 / (sigma * sqrt(2.0 * 3.14159265358979323846));
  double acc = 0.0;
  for (int k = 0; k < scan; ++k) {
    const double x = ang[i] - ang[b0 + k];
    const double g = norm * exp(-0.5 * (x * x) / (sigma * sigma));
    acc += f2[(size_t)(b0 + k) * nb + b] * g * d;
  }
  out[(size_t)i * nb + b] = acc;
}

void launch_rocking_convolution(const double* ang, const double* f2, int rows, int scan, int nb,
                                double omega, double* out, cudaStream_t st) {
  const double sigma = 0.5 * omega / std::sqrt(2.0 * std::log(2.0));
  dim3 grid(ceil_div(nb, 128), rows);
  k_rocking_convolution<<<grid, 128, 0, st>>>(ang, f2, rows, scan, nb, sigma, out);
}

}  // namespace trhepd
