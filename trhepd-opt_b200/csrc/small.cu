// Fused small-beam RKN integration (hp_int_spa, sim-trhepd-rheed/src/surf_prkn.f90:278-330).
//
// For N <= 64 beams a whole angle fits one SM: Q = X^H, P = Y^H and the stage
// matrix (NP x NP complex each, NP = N rounded up to 16) stay in shared memory
// for all s*ns stages, so the solve is one launch (one CTA per angle) instead of
// several launches per stage.  Per stage:
//   * the next stage column's matrix entries are loaded into registers (one fixed
//     set of (k, j) positions per thread, beam-pair indices held in registers)
//     while the current product runs;
//   * the product Q V runs on the FP64 tensor cores (mma.sync m16n8k4, 4 real
//     MMAs per complex product), one warp per 16 rows x NP/2 columns;
//   * the epilogue is the RKN update of the stacked path: P += cb (Q V + Q o D_a),
//     Q <- Q + ca P (the identity stages Q = I are elementwise);
//   * at the end of a slice the renormalisation (policy 0: Gershgorin estimate
//     cond_est, matcomp.f90:498-528, > 1e3; policy 1: every `interval` slices;
//     always on the last) is an in-place Gauss-Jordan of [Q | P] with partial
//     pivoting on max |re| + |im| (matAbdivB, matcomp.f90:53-69), then Q = I.
// The stage order, merged half kicks and coefficients are those of run_rkn.
// One launch can carry several problems (their own tables, beam counts up to
// the launch's NP, slice counts and renormalisation intervals): each CTA finds
// its problem in the launch parameters.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>

#include "small.h"
#include "launch_attr.h"

namespace trhepd {
namespace fused {

template <int NP>
struct Cfg {
  static constexpr int WARPS = NP / 8;              // NP/16 row tiles x 2 column halves
  static constexpr int THREADS = 32 * WARPS;
  static constexpr int QSTR = NP + 4;               // 4 mod 8 complex: conflict-free A reads
  static constexpr int PSTR = NP + 4;
  static constexpr int VSTR = NP + 2;               // 2 mod 8 complex: conflict-free B reads
  static constexpr int NT8 = NP / 16;               // 8-wide column tiles per warp
  static constexpr int GATHER = NP * NP / THREADS;  // stage-matrix entries per thread
  static constexpr size_t SMEM = (size_t)(NP * QSTR + NP * PSTR + NP * VSTR) * sizeof(cd);
};

__device__ __forceinline__ void fdmma(double& c0, double& c1, double& c2, double& c3, double a0,
                                      double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
      : "d"(a0), "d"(a1), "d"(b0));
}

template <int NP>
__global__ void __launch_bounds__(Cfg<NP>::THREADS)
    k_fused_rkn(const __grid_constant__ FusedLaunch L) {
  using C = Cfg<NP>;
  // this CTA's problem: the last whose first CTA is <= blockIdx.x
  int pi = 0;
  for (int q = 1; q < L.nprob; ++q)
    if (L.p[q].first_cta <= (int)blockIdx.x) pi = q;
  const FusedProblem& a = L.p[pi];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cd* Qs = reinterpret_cast<cd*>(smem_raw);
  cd* Ps = Qs + NP * C::QSTR;
  cd* Vs = Ps + NP * C::PSTR;
  __shared__ double red_d[2][C::WARPS];
  __shared__ int piv_sh, renorm_sh;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int n = a.n, ld = a.ld, ang = blockIdx.x - a.first_cta;
  cd* Qg = a.Q + (size_t)ang * n * ld;
  cd* Pg = a.P + (size_t)ang * n * ld;
  const cd* Dg = a.D + (size_t)ang * ld;

  for (int e = tid; e < NP * NP; e += C::THREADS) {
    const int i = e / NP, j = e % NP;
    cd q = cd{0.0, 0.0}, p = cd{0.0, 0.0};
    if (i < n && j < n) {
      q = Qg[(size_t)i * ld + j];
      p = Pg[(size_t)i * ld + j];
    }
    Qs[i * C::QSTR + j] = q;
    Ps[i * C::PSTR + j] = p;
  }
  // this thread's stage-matrix positions: table index (>= 0), -2 diagonal, -1 zero
  int pidx[C::GATHER];
  unsigned upper = 0;
#pragma unroll
  for (int m = 0; m < C::GATHER; ++m) {
    const int e = tid + m * C::THREADS, k = e / NP, j = e % NP;
    pidx[m] = -1;
    if (k < n && j < n) {
      if (k == j) {
        pidx[m] = -2;
      } else {
        pidx[m] = a.pair[k * n + j];
        if (k < j) upper |= 1u << m;
      }
    }
  }
  // row tile and column half of this warp; D of its epilogue columns
  const int m0 = (warp >> 1) * 16, c0 = (warp & 1) * (NP / 2);
  const bool active = m0 < n && c0 < n;
  const int kmax = ((n + 3) / 4) * 4;
  cd dreg[C::NT8][2];
#pragma unroll
  for (int nt = 0; nt < C::NT8; ++nt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int j = c0 + nt * 8 + 2 * t + h;
      dreg[nt][h] = (j < n) ? Dg[j] : cd{0.0, 0.0};
    }

  cd vbuf[C::GATHER];
  auto load_col = [&](int col) {
    const TableEntry* tc = a.table + (size_t)col * a.nv;
#pragma unroll
    for (int m = 0; m < C::GATHER; ++m) {
      const int p = pidx[m];
      cd v = cd{0.0, 0.0};
      if (p >= 0) {
        v = ((upper >> m) & 1u) ? -conj(tc[p].u) : -tc[p].w;
      } else if (p == -2) {
        v = -conj(tc[0].u);
      }
      vbuf[m] = v;
    }
  };
  auto store_col = [&]() {
#pragma unroll
    for (int m = 0; m < C::GATHER; ++m) {
      const int e = tid + m * C::THREADS;
      Vs[(e / NP) * C::VSTR + (e % NP)] = vbuf[m];
    }
  };
  // P += cb (V + diag(D)), Q = I + ca P  (stage with Q = I)
  auto identity_stage = [&](double cb, double ca) {
    for (int e = tid; e < n * n; e += C::THREADS) {
      const int i = e / n, j = e % n;
      cd m = Vs[i * C::VSTR + j];
      if (i == j) m = m + Dg[j];
      const cd p = Ps[i * C::PSTR + j] + cb * m;
      Ps[i * C::PSTR + j] = p;
      cd q = ca * p;
      if (i == j) q.x += 1.0;
      Qs[i * C::QSTR + j] = q;
    }
  };
  // P += cb (Q V + Q o D), Q <- Q + ca P; the caller has synchronised; returns
  // after the product phase's barrier, with the update written (no trailing barrier)
  auto product_stage = [&](double cb, double ca) {
    double cr[C::NT8][4], ci[C::NT8][4];
#pragma unroll
    for (int nt = 0; nt < C::NT8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) cr[nt][e] = ci[nt][e] = 0.0;
    if (active) {
      for (int k = 0; k < kmax; k += 4) {
        const cd a0 = Qs[(m0 + g) * C::QSTR + k + t];
        const cd a1 = Qs[(m0 + g + 8) * C::QSTR + k + t];
#pragma unroll
        for (int nt = 0; nt < C::NT8; ++nt) {
          const cd b = Vs[(k + t) * C::VSTR + c0 + nt * 8 + g];
          double* R = cr[nt];
          double* I = ci[nt];
          fdmma(R[0], R[1], R[2], R[3], a0.x, a1.x, b.x);
          fdmma(R[0], R[1], R[2], R[3], -a0.y, -a1.y, b.y);
          fdmma(I[0], I[1], I[2], I[3], a0.x, a1.x, b.y);
          fdmma(I[0], I[1], I[2], I[3], a0.y, a1.y, b.x);
        }
      }
    }
    __syncthreads();  // every read of Q and V done
    if (active) {
#pragma unroll
      for (int nt = 0; nt < C::NT8; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int i = m0 + g + ((e >= 2) ? 8 : 0);
          const int j = c0 + nt * 8 + 2 * t + (e & 1);
          if (i < n && j < n) {
            const cd q = Qs[i * C::QSTR + j];
            const cd acc = cd{cr[nt][e], ci[nt][e]} + q * dreg[nt][e & 1];
            const cd p = Ps[i * C::PSTR + j] + cb * acc;
            Ps[i * C::PSTR + j] = p;
            Qs[i * C::QSTR + j] = q + ca * p;
          }
        }
    }
  };
  // Gershgorin estimate of Q (cond_est) > 1e3
  auto needs_renorm = [&]() -> bool {
    double mn = INFINITY, mx = 0.0;
    if (tid < n) {
      const int j = tid;
      double tsum = 0.0;
      for (int i = 0; i < n; ++i)
        if (i != j) {
          const cd v = Qs[i * C::QSTR + j];
          tsum = tsum + sqrt(v.x * v.x + v.y * v.y);
        }
      const cd dj = Qs[j * C::QSTR + j];
      const double ad = hypot(dj.x, dj.y);
      mn = ad - tsum;
      mx = ad + tsum;
    }
    for (int o = 16; o > 0; o >>= 1) {
      mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0) {
      red_d[0][warp] = mn;
      red_d[1][warp] = mx;
    }
    __syncthreads();
    if (tid == 0) {
      for (int w = 1; w < C::WARPS; ++w) {
        mn = fmin(mn, red_d[0][w]);
        mx = fmax(mx, red_d[1][w]);
      }
      const cd a11 = Qs[0];
      mx = fmax(mx, hypot(a11.x, a11.y));
      const double d = (mn < 0.0) ? 1e100 : mx / mn;
      renorm_sh = d > 1e3;
    }
    __syncthreads();
    return renorm_sh != 0;
  };
  // [Q | P] -> [I | Q^{-1} P]
  auto gauss_jordan = [&]() {
    for (int c = 0; c < n; ++c) {
      if (warp == 0) {
        double best = -1.0;
        int bi = n;
        for (int r = c + lane; r < n; r += 32) {
          const double v = cabs1(Qs[r * C::QSTR + c]);
          if (v > best) {
            best = v;
            bi = r;
          }
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ov > best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
          }
        }
        if (lane == 0) {
          piv_sh = bi;
          if (!(best > 0.0)) atomicOr(a.status, kStatusZeroPivot);
        }
      }
      __syncthreads();
      const int piv = piv_sh;
      if (piv != c)
        for (int j = tid; j < 2 * n; j += C::THREADS) {
          if (j < n) {
            if (j >= c) {
              const cd x = Qs[c * C::QSTR + j];
              Qs[c * C::QSTR + j] = Qs[piv * C::QSTR + j];
              Qs[piv * C::QSTR + j] = x;
            }
          } else {
            const int jp = j - n;
            const cd x = Ps[c * C::PSTR + jp];
            Ps[c * C::PSTR + jp] = Ps[piv * C::PSTR + jp];
            Ps[piv * C::PSTR + jp] = x;
          }
        }
      __syncthreads();
      const cd inv = cdiv(cd{1.0, 0.0}, Qs[c * C::QSTR + c]);
      const int wq = n - c - 1, W = wq + n;
      for (int e = tid; e < n * W; e += C::THREADS) {
        const int r = e / W, jj = e - r * W;
        if (r == c) continue;
        const cd f = Qs[r * C::QSTR + c] * inv;
        if (jj < wq) {
          const int j = c + 1 + jj;
          Qs[r * C::QSTR + j] = Qs[r * C::QSTR + j] - f * Qs[c * C::QSTR + j];
        } else {
          const int j = jj - wq;
          Ps[r * C::PSTR + j] = Ps[r * C::PSTR + j] - f * Ps[c * C::PSTR + j];
        }
      }
      __syncthreads();
      for (int j = tid; j < W; j += C::THREADS) {
        if (j < wq)
          Qs[c * C::QSTR + c + 1 + j] = Qs[c * C::QSTR + c + 1 + j] * inv;
        else
          Ps[c * C::PSTR + j - wq] = Ps[c * C::PSTR + j - wq] * inv;
      }
      __syncthreads();
    }
    for (int e = tid; e < n * n; e += C::THREADS) {
      const int i = e / n, j = e % n;
      Qs[i * C::QSTR + j] = cd{(i == j) ? 1.0 : 0.0, 0.0};
    }
  };

  const int s = L.s, ns = a.ns;
  const double dz = a.dz;
  load_col(0);
  store_col();
  __syncthreads();
  load_col(1);
  identity_stage(L.bab[0] * dz, L.bab[1] * dz);
  __syncthreads();
  store_col();
  __syncthreads();
  for (int l = 1; l <= ns; ++l) {
    for (int k = (l == 1) ? 2 : 1; k <= s; ++k) {
      const int col = s * (l - 1) + k - 1;
      const double ca = L.bab[2 * k - 1] * dz;
      // k == 1 merges the end-of-slice half kick of slice l-1 with the first kick
      const double cb = (k == 1) ? 2.0 * L.bab[0] * dz : L.bab[2 * k - 2] * dz;
      load_col(col + 1);  // the next stage's matrix (the last column after slice ns)
      product_stage(cb, ca);
      store_col();        // V is no longer read: the next stage's matrix goes in
      __syncthreads();
    }
    const bool last = l == ns;
    bool renorm = last;
    if (!last) renorm = (L.policy == 0) ? needs_renorm() : (l % a.interval) == 0;
    if (renorm) {
      gauss_jordan();
      __syncthreads();
    }
  }
  // final half kick with Q = I: P += b1 dz M(end)
  identity_stage(L.bab[0] * dz, 0.0);
  __syncthreads();
  for (int e = tid; e < n * n; e += C::THREADS) {
    const int i = e / n, j = e % n;
    Qg[(size_t)i * ld + j] = Qs[i * C::QSTR + j];
    Pg[(size_t)i * ld + j] = Ps[i * C::PSTR + j];
  }
}

template <int NP>
void launch(const FusedLaunch& L, cudaStream_t st) {
  using C = Cfg<NP>;
  static SmemOptIn attr;
  attr.ensure((const void*)k_fused_rkn<NP>, C::SMEM);
  k_fused_rkn<NP><<<L.total_ctas, C::THREADS, C::SMEM, st>>>(L);
}

}  // namespace fused

int launch_fused_rkn(const FusedLaunch& L, cudaStream_t st) {
  if (L.nprob < 1 || L.nprob > kFusedMaxProblems || L.s < 1 || L.s > 11)
    throw std::invalid_argument("fused integration: bad launch");
  int nmax = 0, ctas = 0;
  for (int q = 0; q < L.nprob; ++q) {
    const FusedProblem& a = L.p[q];
    if (a.n < 2 || a.n > kFusedMaxBeams || a.ns < 1 || a.interval < 1 || a.nang < 1 ||
        a.first_cta != ctas)
      throw std::invalid_argument("fused integration: unsupported problem");
    ctas += a.nang;
    nmax = std::max(nmax, a.n);
  }
  if (ctas != L.total_ctas) throw std::invalid_argument("fused integration: CTA count");
  if (nmax <= 16)
    fused::launch<16>(L, st);
  else if (nmax <= 32)
    fused::launch<32>(L, st);
  else if (nmax <= 48)
    fused::launch<48>(L, st);
  else
    fused::launch<64>(L, st);
  return 1;
}

}  // namespace trhepd
