// Split-precision stage product on the 5th-generation tensor cores (sm_100a).
//
// The integrator stage (surf_prkn.f90:222-276, batched over angles)
//     P += cb * Q M,   M = Voff + diag(vd + d_a),   Q <- Q + ca * P
// is formed as
//     Q M = Qoff Voff  +  diag(q) Voff  +  Q diag(vd + d_a)
// where Qoff / Voff are Q and the shared potential matrix with their diagonals
// removed and q is Q's diagonal.  The last two terms are exact FP64 work in the
// epilogue; Qoff Voff runs on tcgen05 from BF16 slices:
//
//   * every row r of Qoff is scaled by a power of two 2^-e_r (row maximum), every
//     column j of Voff by 2^-f_j, and the scaled values are cut into S signed
//     base-256 digits d_s in [-128, 128] with rounding; slice s holds d_s * 2^-8s,
//     so each slice is exact in BF16 and a slice pair (s, t) carries its weight;
//   * complex is handled as a real product with interleaved components:
//     A = [Re Q, Im Q] per column pair, B^T rows (Re-out, Im-out) per column pair;
//   * the slice pairs with s + t < S are issued into three FP32 TMEM accumulators
//     (s+t = 0, s+t = 1, s+t >= 2).  The first two hold integer sums well inside
//     FP32's 24-bit exact range, so only the small third one rounds;
//   * the epilogue combines the accumulators in FP64, rescales by 2^(e_r + f_j - 14)
//     and performs the RKN update with the exact diagonal terms.
//
// Layouts: A slices [S][R][KR] and B^T slices [S][NR][KR], BF16, K-major, loaded by
// TMA with 64-byte swizzle in 32-element k-blocks; one CTA computes 128 rows x
// 128 real columns (64 complex); warp 0 issues TMA, warp 1 issues MMA, warps 2-5
// drain TMEM.  All waits are bounded and report kStatusTimeout instead of hanging.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "kernels.h"
#include "launch_attr.h"
#include "split_gemm.h"

namespace trhepd {
namespace split {

constexpr int BM = 128;               // UMMA M: stacked rows per CTA
constexpr int NT = 128;               // UMMA N: real output columns per CTA (64 complex)
constexpr int NC = NT / 2;            // complex columns per CTA
constexpr int BK = 32;                // real k per pipeline stage (64-byte rows)
constexpr int NACC = 3;
constexpr int TMEM_COLS = 512;
constexpr int THREADS = 192;
constexpr int A_SLICE_BYTES = BM * BK * 2;
constexpr int B_SLICE_BYTES = NT * BK * 2;
constexpr int EPI_STRIDE = NC + 1;    // complex elements per staged row (odd: conflict-free)
constexpr uint64_t kWaitNs = 2000000000ull;  // bounded waits give up after ~2 s
constexpr double kDigitHeadroom = 1.0 + 1.0 / 128;  // INT8 exponents: |d_0| <= 127

__host__ __device__ constexpr int stages_for(int S) { return S <= 4 ? 3 : 2; }
__host__ __device__ constexpr size_t stage_bytes(int S) {
  return (size_t)S * (A_SLICE_BYTES + B_SLICE_BYTES);
}
inline size_t smem_bytes(int S) {
  size_t pipe = stages_for(S) * stage_bytes(S);
  size_t epi = (size_t)BM * EPI_STRIDE * sizeof(cd);
  return 1024 + (pipe > epi ? pipe : epi);
}

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on phase `parity`; returns false once ~2 s have passed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t a = smem_u32(bar);
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 1023) == 1023 && globaltimer() - t0 > kWaitNs) return false;
  }
}
__device__ __forceinline__ void tma_load_3d(const CUtensorMap* map, uint64_t* bar, void* dst,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, 64-byte swizzle, 8-row groups 512 B apart.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);       // start address
  d |= (uint64_t)1 << 16;                       // leading byte offset (16 B units)
  d |= (uint64_t)(512 >> 4) << 32;              // stride byte offset
  d |= (uint64_t)1 << 46;                       // descriptor version
  d |= (uint64_t)4 << 61;                       // SWIZZLE_64B
  return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = NT.
__host__ __device__ constexpr uint32_t instr_desc() {
  return (1u << 4)                      // D format F32
         | (1u << 7) | (1u << 10)       // A, B format BF16
         | ((uint32_t)(NT >> 3) << 17)  // N
         | ((uint32_t)(BM >> 4) << 24); // M
}

struct EpiArgs {
  const cd* Q;
  cd* P;
  cd* Qo;
  const cd* V;         // Voff (kpad + 1 rows, the last one holds the dropped diagonal)
  const cd* D;         // -conj(gamma^2) per angle (nang x ld)
  const int* erow;     // row exponents
  const int* fcol;     // column exponents (complex columns)
  unsigned* status;
  int rows, n, ld, kpad, S;
  double cb, ca;
  // stacked problems (INT8 kernel): problem b owns rows [b rows_b, (b+1) rows_b),
  // its stage matrix at V + b vstride and its column exponents at fcol + b fstride;
  // tpp row tiles per problem
  int rows_b = 0, fstride = 0, tpp = 0;
  long long vstride = 0;
  int* tile_counter = nullptr;  // INT8 kernel: {next tile, finished CTAs}, zero between launches
};

// ------------------------------------------------------------ slicing kernels
// Digits of x * 2^(7 - e): d0 = rint(y), y <- (y - d0) * 256, ...; slice s = d_s 2^-8s.
template <int S>
__device__ __forceinline__ void digits(double x, int e, float* out) {
  double y = ldexp(x, 7 - e);
#pragma unroll
  for (int s = 0; s < S; ++s) {
    double d = rint(y);
    out[s] = ldexpf((float)d, -8 * s);
    y = (y - d) * 256.0;
  }
}

// One warp per stacked row: exponent of the off-diagonal row maximum, then the
// S interleaved (Re, Im) slices of the row.
template <int S>
__global__ void k_slice_rows(const cd* __restrict__ Q, int rows, int n, int ld, int kr,
                             __nv_bfloat162* __restrict__ A, int* __restrict__ erow) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const int r = warp, i = r % n;
  const cd* q = Q + (size_t)r * ld;
  double m = 0.0;
  for (int k = lane; k < n; k += 32)
    if (k != i) m = fmax(m, fmax(fabs(q[k].x), fabs(q[k].y)));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  int e = 0;
  if (m > 0.0) frexp(m, &e);  // m < 2^e
  if (lane == 0) erow[r] = e;
  const int kc = kr / 2;
  for (int k = lane; k < kc; k += 32) {
    cd v = (k < n && k != i) ? q[k] : cd{0.0, 0.0};
    float dr[S], di[S];
    digits<S>(v.x, e, dr);
    digits<S>(v.y, e, di);
#pragma unroll
    for (int s = 0; s < S; ++s)
      A[((size_t)s * rows + r) * kc + k] = __floats2bfloat162_rn(dr[s], di[s]);
  }
}

// Column exponents of Voff: 32 columns per block, the 8 warps split the rows
// (lanes read consecutive columns), then a shared-memory maximum; the exponent is
// that of the maximum times `headroom` (1, or kDigitHeadroom for INT8 digits).
__global__ void __launch_bounds__(256) k_col_exponents(const cd* __restrict__ V, int n, int ld,
                                                       double headroom, int* __restrict__ fcol) {
  __shared__ double red[8][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + lane;
  double m = 0.0;
  if (j < n)
    for (int k = w; k < n; k += 8) {
      cd v = V[(size_t)k * ld + j];
      m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
  red[w][lane] = m;
  __syncthreads();
  if (w == 0 && j < n) {
    for (int q = 1; q < 8; ++q) m = fmax(m, red[q][lane]);
    int e = 0;
    if (m > 0.0) frexp(m * headroom, &e);
    fcol[j] = e;
  }
}

// B^T slices: row 2j (Re-out) = [Vr(k,j), -Vi(k,j)]_k, row 2j+1 (Im-out) = [Vi, Vr]_k.
template <int S>
__global__ void k_slice_cols(const cd* __restrict__ V, int n, int ld, int kc, int nrows,
                             const int* __restrict__ fcol, __nv_bfloat162* __restrict__ B) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (k >= kc || j >= n) return;
  cd v = (k < n) ? V[(size_t)k * ld + j] : cd{0.0, 0.0};
  const int e = fcol[j];
  float dr[S], di[S];
  digits<S>(v.x, e, dr);
  digits<S>(v.y, e, di);
#pragma unroll
  for (int s = 0; s < S; ++s) {
    B[((size_t)s * nrows + 2 * j) * kc + k] = __floats2bfloat162_rn(dr[s], -di[s]);
    B[((size_t)s * nrows + 2 * j + 1) * kc + k] = __floats2bfloat162_rn(di[s], dr[s]);
  }
}

// ------------------------------------------------------------ tcgen05 GEMM + epilogue
template <int S>
__global__ void __launch_bounds__(THREADS, 1)
    k_split_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                 EpiArgs ep, int nkb) {
  constexpr int STAGES = stages_for(S);
  // an earlier launch gave up on a wait: skip the work, the host reports it
  if (*(volatile unsigned*)ep.status & kStatusTimeout) return;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[3], empty_bar[3], done_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int fexp_sh[NC];
  __shared__ int abort_sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM;
  const int n0 = blockIdx.x * NT;        // real column
  const int j0 = blockIdx.x * NC;        // complex column

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    abort_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  for (int t = threadIdx.x; t < NC; t += THREADS) {
    int j = j0 + t;
    fexp_sh[t] = (j < ep.n) ? ep.fcol[j] : 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  const size_t sbytes = stage_bytes(S);

  if (warp == 0) {
    // ---------------- TMA producer
    if (lane == 0) {
      for (int kb = 0; kb < nkb; ++kb) {
        const int st = kb % STAGES, round = kb / STAGES;
        if (round > 0 && !mbar_wait(&empty_bar[st], (round - 1) & 1)) {
          atomicOr(ep.status, kStatusTimeout);
          abort_sh = 1;
          break;
        }
        if (abort_sh) break;
        unsigned char* sa = smem + st * sbytes;
        unsigned char* sb = sa + S * A_SLICE_BYTES;
        mbar_expect_tx(&full_bar[st], (uint32_t)sbytes);
#pragma unroll
        for (int s = 0; s < S; ++s) {
          tma_load_3d(&tmA, &full_bar[st], sa + s * A_SLICE_BYTES, kb * BK, m0, s);
          tma_load_3d(&tmB, &full_bar[st], sb + s * B_SLICE_BYTES, kb * BK, n0, s);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = instr_desc();
      bool started[NACC] = {false, false, false};
      for (int kb = 0; kb < nkb; ++kb) {
        const int st = kb % STAGES, round = kb / STAGES;
        if (!mbar_wait(&full_bar[st], round & 1)) {
          atomicOr(ep.status, kStatusTimeout);
          abort_sh = 1;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + st * sbytes);
        const uint32_t sb = sa + S * A_SLICE_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
#pragma unroll
          for (int s = 0; s < S; ++s) {
#pragma unroll
            for (int t = 0; t < S - s; ++t) {
              const int acc = (s + t < 2) ? s + t : 2;
              const uint64_t ad = sw64_desc(sa + s * A_SLICE_BYTES + kk * 32);
              const uint64_t bd = sw64_desc(sb + t * B_SLICE_BYTES + kk * 32);
              tc_mma(tmem + acc * NT, ad, bd, idesc, started[acc] ? 1u : 0u);
              started[acc] = true;
            }
          }
        }
        tc_commit(&empty_bar[st]);  // frees the stage once these MMAs complete
      }
      tc_commit(&done_bar);
    }
  } else {
    // ---------------- TMEM drain (warps 2..5): rows 32*(warp%4) .. +31
    const int q4 = warp & 3;
    const int rl = q4 * 32 + lane;  // local row of this thread
    const int r = m0 + rl;
    const bool ok = mbar_wait(&done_bar, 0);
    if (!ok) atomicOr(ep.status, kStatusTimeout);
    tc_fence_after();
    cd* stage_out = reinterpret_cast<cd*>(smem);
    const int er = (r < ep.rows) ? ep.erow[r] : 0;
    const uint32_t lane_base = tmem + ((uint32_t)(q4 * 32) << 16);
    for (int c = 0; c < NT / 16; ++c) {
      uint32_t a0[16], a1[16], a2[16];
      tmem_ld16(lane_base + 0 * NT + c * 16, a0);
      tmem_ld16(lane_base + 1 * NT + c * 16, a1);
      tmem_ld16(lane_base + 2 * NT + c * 16, a2);
      tmem_wait_ld();
#pragma unroll
      for (int e2 = 0; e2 < 8; ++e2) {
        const int jl = c * 8 + e2;  // local complex column
        const int sc = er + fexp_sh[jl] - 14;
        double re = (double)__uint_as_float(a2[2 * e2]) + (double)__uint_as_float(a1[2 * e2]) +
                    (double)__uint_as_float(a0[2 * e2]);
        double im = (double)__uint_as_float(a2[2 * e2 + 1]) +
                    (double)__uint_as_float(a1[2 * e2 + 1]) +
                    (double)__uint_as_float(a0[2 * e2 + 1]);
        stage_out[rl * EPI_STRIDE + jl] = cd{ldexp(re, sc), ldexp(im, sc)};
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  // ---------------- fused FP64 epilogue, coalesced over columns
  if (!abort_sh) {
    const cd* stage_out = reinterpret_cast<const cd*>(smem);
    const cd vd = ep.V[(size_t)ep.kpad * ep.ld];
    for (int rl = warp; rl < BM; rl += THREADS / 32) {
      const int r = m0 + rl;
      if (r >= ep.rows) break;
      const int a = r / ep.n, i = r - a * ep.n;
      const size_t ro = (size_t)r * ep.ld;
      const cd qd = ep.Q[ro + i];
      for (int jl = lane; jl < NC; jl += 32) {
        const int j = j0 + jl;
        if (j >= ep.n) break;
        const cd q = ep.Q[ro + j];
        const cd d = ep.D[(size_t)a * ep.ld + j] + vd;
        const cd acc = stage_out[rl * EPI_STRIDE + jl] + qd * ep.V[(size_t)i * ep.ld + j] + q * d;
        const cd p = ep.P[ro + j] + ep.cb * acc;
        ep.P[ro + j] = p;
        ep.Qo[ro + j] = q + ep.ca * p;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

// ------------------------------------------------------------ persistent form
// One CTA per SM walks the tiles (static stride) with the mainloop and the three
// accumulators of the per-tile form (s+t = 0, 1, >= 2; 384 TMEM columns).  Eight
// epilogue warps (two per TMEM lane quadrant, one per 32-column half) drain a
// finished tile with 16x256b TMEM loads, which hand each lane complex values in
// column-coalesced position (rows t/4 and t/4 + 8 of a 16-row block, complex
// column t%4 of a 4-column group), keep them in registers as scaled FP64 and give
// the TMEM back at once; the MMAs of the next tile then run while the same warps
// perform the HBM-bound RKN update from registers.  The register file is split
// with setmaxnreg: the control warpgroup (TMA, MMA, two idle warps) drops to
// P_REG_CTRL, the two epilogue warpgroups rise to P_REG_EPI.
constexpr int P_THREADS = 384;   // warps 0 TMA, 1 MMA, 2-3 idle, 4-11 epilogue
constexpr int P_EPI_WARPS = 8;
constexpr int P_REG_LAUNCH = 168;  // registers per thread the launch must provide
constexpr int P_REG_CTRL = 40;
constexpr int P_REG_EPI = 232;
static_assert(128 * P_REG_CTRL + 256 * P_REG_EPI <= P_THREADS * P_REG_LAUNCH,
              "setmaxnreg split exceeds the launch's registers");
__host__ __device__ constexpr int pstages_for(int S) { return stages_for(S); }
inline size_t psmem_bytes(int S) { return smem_bytes(S); }

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }
// 2^e as a double: exact bit construction in the normal range, ldexp outside it.
__device__ __forceinline__ double pow2(int e) {
  return (e > -1022 && e < 1023) ? __longlong_as_double((long long)(e + 1023) << 52)
                                 : ldexp(1.0, e);
}
// 16 TMEM lanes x 256 bits: r0, r1 = lane t/4, 32-bit columns 2(t%4), 2(t%4)+1;
// r2, r3 = the same columns of lane t/4 + 8.
__device__ __forceinline__ void tmem_ld_16x256(uint32_t taddr, uint32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.16x256b.x1.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}
// Named barrier of the epilogue warps returning whether any thread passed
// fail != 0, so that all of them take the same branch afterwards.
__device__ __forceinline__ bool epi_any(int fail) {
  uint32_t any;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 q, %1, 0;\n\t"
      "bar.red.or.pred p, 1, %2, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(any)
      : "r"(fail), "n"(32 * P_EPI_WARPS)
      : "memory");
  return any != 0;
}

template <int S>
__global__ void __launch_bounds__(P_THREADS, 1)
    k_split_gemm_p(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   EpiArgs ep, int nkb, int tiles_n, int tiles) {
  constexpr int STAGES = pstages_for(S);
  // an earlier launch gave up on a wait: skip the work, the host reports it
  if (*(volatile unsigned*)ep.status & kStatusTimeout) return;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], tfull, tempty, drain_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh, issued_sh, consumed_sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t sbytes = stage_bytes(S);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&tfull, 1);
    mbar_init(&tempty, P_EPI_WARPS);
    mbar_init(&drain_bar, 1);
    abort_sh = 0;
    issued_sh = 0;
    consumed_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(P_REG_CTRL));
  if (warp == 0) {
    // ---------------- TMA producer
    if (lane == 0) {
      int g = 0;
      bool stop = false;
      for (int tile = blockIdx.x; tile < tiles && !stop; tile += gridDim.x) {
        const int m0 = (tile / tiles_n) * BM, n0 = (tile % tiles_n) * NT;
        for (int kb = 0; kb < nkb; ++kb, ++g) {
          const int st = g % STAGES, round = g / STAGES;
          if (round > 0 && !mbar_wait(&empty_bar[st], (round - 1) & 1)) {
            atomicOr(ep.status, kStatusTimeout);
            abort_sh = 1;
            stop = true;
            break;
          }
          if (ld_volatile(&abort_sh)) {
            stop = true;
            break;
          }
          unsigned char* sa = smem + st * sbytes;
          unsigned char* sb = sa + S * A_SLICE_BYTES;
          mbar_expect_tx(&full_bar[st], (uint32_t)sbytes);
#pragma unroll
          for (int s = 0; s < S; ++s) {
            tma_load_3d(&tmA, &full_bar[st], sa + s * A_SLICE_BYTES, kb * BK, m0, s);
            tma_load_3d(&tmB, &full_bar[st], sb + s * B_SLICE_BYTES, kb * BK, n0, s);
          }
        }
      }
      issued_sh = g;
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = instr_desc();
      int g = 0, it = 0;
      bool stop = false;
      for (int tile = blockIdx.x; tile < tiles && !stop; tile += gridDim.x, ++it) {
        // the accumulators of the previous tile must have been drained
        if (it > 0 && !mbar_wait(&tempty, (it - 1) & 1)) {
          atomicOr(ep.status, kStatusTimeout);
          abort_sh = 1;
          break;
        }
        tc_fence_after();
        bool started[NACC] = {false, false, false};
        for (int kb = 0; kb < nkb; ++kb, ++g) {
          const int st = g % STAGES, round = g / STAGES;
          if (!mbar_wait(&full_bar[st], round & 1)) {
            atomicOr(ep.status, kStatusTimeout);
            abort_sh = 1;
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + st * sbytes);
          const uint32_t sb = sa + S * A_SLICE_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
#pragma unroll
              for (int t = 0; t < S - s; ++t) {
                const int acc = (s + t < 2) ? s + t : 2;
                const uint64_t ad = sw64_desc(sa + s * A_SLICE_BYTES + kk * 32);
                const uint64_t bd = sw64_desc(sb + t * B_SLICE_BYTES + kk * 32);
                tc_mma(tmem + acc * NT, ad, bd, idesc, started[acc] ? 1u : 0u);
                started[acc] = true;
              }
            }
          }
          tc_commit(&empty_bar[st]);
        }
        if (stop) break;
        tc_commit(&tfull);
      }
      consumed_sh = g;
      // no MMA may still be running when the TMEM is released
      tc_commit(&drain_bar);
      if (!mbar_wait(&drain_bar, 0)) atomicOr(ep.status, kStatusTimeout);
    }
  }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(P_REG_EPI));
    // ---------------- epilogue warps 4..11
    const int q4 = warp & 3;                 // TMEM lane quadrant
    const int half = (warp - 4) >> 2;        // 32-complex-column half of the tile
    const int t0 = lane & 3, t1 = lane >> 2;
    const cd vd = ep.V[(size_t)ep.kpad * ep.ld];
    int it = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++it) {
      const int m0 = (tile / tiles_n) * BM + q4 * 32;          // first row of this quadrant
      const int jh = (tile % tiles_n) * NC + half * (NC / 2);  // first complex column
      // this lane's rows m0 + 16h + 8u + t1 and columns jh + 4g + t0
      int er[2][2], ra[2][2], ri[2][2];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int r = m0 + 16 * h + 8 * u + t1;
          er[h][u] = 0;
          ra[h][u] = 0;
          ri[h][u] = 0;
          if (r < ep.rows) {
            er[h][u] = ep.erow[r];
            ra[h][u] = r / ep.n;
            ri[h][u] = r - ra[h][u] * ep.n;
          }
        }
      int fc[8];
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        const int j = jh + 4 * g + t0;
        fc[g] = (j < ep.n) ? ep.fcol[j] : 0;
      }
      const bool ok = mbar_wait(&tfull, it & 1);
      if (epi_any(!ok)) {  // uniform across the epilogue warps
        if (!ok) atomicOr(ep.status, kStatusTimeout);
        abort_sh = 1;
        break;
      }
      tc_fence_after();
      // drain: (acc2 + acc1) + acc0 in FP64 (the order of the per-tile form),
      // scaled exactly by 2^(e_r + f_j - 14)
      cd vals[8][2][2];
#pragma unroll
      for (int g = 0; g < 8; ++g)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t taddr = tmem + ((uint32_t)(q4 * 32 + 16 * h) << 16) +
                                 (uint32_t)(2 * (half * (NC / 2) + 4 * g));
          uint32_t a2[4], a1[4], a0[4];
          tmem_ld_16x256(taddr + 2 * NT, a2);
          tmem_ld_16x256(taddr + 1 * NT, a1);
          tmem_ld_16x256(taddr + 0 * NT, a0);
          tmem_wait_ld();
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const double re = (double)__uint_as_float(a2[2 * u]) +
                              (double)__uint_as_float(a1[2 * u]) +
                              (double)__uint_as_float(a0[2 * u]);
            const double im = (double)__uint_as_float(a2[2 * u + 1]) +
                              (double)__uint_as_float(a1[2 * u + 1]) +
                              (double)__uint_as_float(a0[2 * u + 1]);
            const double sc = pow2(er[h][u] + fc[g] - 14);
            vals[g][h][u] = cd{re * sc, im * sc};
          }
        }
      // the accumulators are in registers: let the next tile's MMAs start
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty);
      // RKN update from registers; each warp access covers 8 rows x 4 columns
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        const int j = jh + 4 * g + t0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          cd qv[2], pv[2], qd[2], vv[2], dv[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int r = m0 + 16 * h + 8 * u + t1;
            if (r < ep.rows && j < ep.n) {
              const size_t ro = (size_t)r * ep.ld;
              qv[u] = ep.Q[ro + j];
              pv[u] = ep.P[ro + j];
              qd[u] = ep.Q[ro + ri[h][u]];
              vv[u] = ep.V[(size_t)ri[h][u] * ep.ld + j];
              dv[u] = ep.D[(size_t)ra[h][u] * ep.ld + j];
            }
          }
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int r = m0 + 16 * h + 8 * u + t1;
            if (r < ep.rows && j < ep.n) {
              const size_t ro = (size_t)r * ep.ld;
              const cd acc = vals[g][h][u] + qd[u] * vv[u] + qv[u] * (dv[u] + vd);
              const cd p = pv[u] + ep.cb * acc;
              ep.P[ro + j] = p;
              ep.Qo[ro + j] = qv[u] + ep.ca * p;
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    // bulk copies issued but never consumed (only after a timeout) must land
    // before the CTA exits
    for (int g = consumed_sh; g < issued_sh; ++g)
      if (!mbar_wait(&full_bar[g % STAGES], (g / STAGES) & 1)) break;
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

// ------------------------------------------------------------ INT8 form
// The same stage product from signed 8-bit digits on kind::i8 with exact INT32
// accumulation (twice the BF16 MMA rate).  A row (column) whose largest entry is m
// gets the exponent e of m (1 + 2^-7), so |x| < 2^e (1 - 2^-8) for its entries;
// each entry is rounded once to the integer
//     X = rint(x 2^(7 - e + 8(S-1)))
// and written in balanced base 256, X = sum_s d_s 256^(S-1-s), d_s in [-128, 127]
// for s >= 1; the headroom keeps |d_0| <= 127.  So x = 2^(e-7) sum_s d_s 2^-8s up
// to half a unit of the last digit.  The slice pairs with s + t = L go to INT32
// accumulator L (L < S, S x NT(S) TMEM columns); every sum is exact (|acc_L| <=
// S * 2^14 * K, below 2^31 for K < 16384), and the epilogue forms
// sum_L 2^-8L acc_L in FP64 and scales it by 2^(e_r + f_j - 14).  S = 3..6: each
// digit adds 8 bits (31 bits at S = 4, 47 at S = 6); tiles narrow from 128 to 96
// and 80 real columns at S = 5, 6 so that the S levels fit the TMEM.
namespace i8 {
constexpr int BK = 64;                     // int8 k per pipeline stage (64-byte rows)
constexpr int STAGES = 2;                  // pipeline stages of S A- and S B-slices
constexpr int A_SLICE_BYTES = BM * BK;     // 8 KB
// Real output columns per tile: the S accumulator levels of a tile must fit the
// 512 TMEM columns (S * NT <= 512), and NT is a multiple of 16 for M = 128.
__host__ __device__ constexpr int nt_for(int S) { return S <= 4 ? 128 : (S == 5 ? 96 : 80); }
__host__ __device__ constexpr int nc_for(int S) { return nt_for(S) / 2; }
__host__ __device__ constexpr int b_slice_bytes(int S) { return nt_for(S) * BK; }
__host__ __device__ constexpr size_t stage_bytes(int S) {
  return (size_t)S * (A_SLICE_BYTES + b_slice_bytes(S));
}
// Epilogue tables: the per-angle diagonal D of the angles a tile's rows belong to,
// at most kDTabBytes per tile (two buffers, so that filling the next tile's table
// never overlaps reads of the current one).
constexpr int kDTabBytes = 4096;
// Epilogue load ring: the RKN update reads every state entry (Q and P) once, so the
// epilogue warps stream them from HBM into shared memory with cp.async several
// update steps ahead of their use, across tile boundaries, holding no registers for
// the loads in flight.  One slot = Q and P of each epilogue lane's two rows of one
// step (16 bytes each): 16 KB.  As many slots as the shared memory left beside
// the pipeline allows.
constexpr int kRingItems = 4;
constexpr size_t kSlotBytes = (size_t)kRingItems * 8 /* epilogue warps */ * 32 * 16;
constexpr size_t kSmemCap = 232448 - 512;  // per-block opt-in limit, less static shared
__host__ __device__ constexpr int ring_slots(int S) {
  return (int)((kSmemCap - 1024 - STAGES * stage_bytes(S) - 2 * kDTabBytes) / kSlotBytes) > 6
             ? 6
             : (int)((kSmemCap - 1024 - STAGES * stage_bytes(S) - 2 * kDTabBytes) / kSlotBytes);
}
inline size_t smem_bytes(int S) {
  return 1024 + STAGES * stage_bytes(S) + 2 * kDTabBytes + ring_slots(S) * kSlotBytes;
}
// Steps ahead at which the epilogue loads the stage matrix entries it needs
// (registers: the narrower tiles of S = 5, 6 leave room for more).
__host__ __device__ constexpr int v_ahead(int S) { return S <= 4 ? 1 : (S == 5 ? 2 : 3); }
static_assert(ring_slots(3) >= 3 && ring_slots(4) >= 3 && ring_slots(5) >= 3 &&
                  ring_slots(6) >= 3,
              "epilogue ring needs at least three slots");
}  // namespace i8

// 16-byte global -> shared copy, cached in L2 only (the state is read once).
__device__ __forceinline__ void cp_async_16(uint32_t saddr, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// An INT32 accumulator value as a double without the conversion unit: the bits
// 0x43380000:(a + 2^31) form 2^52 + 2^51 + 2^31 + a exactly, from which the
// constant is subtracted exactly (magic-number conversion).
__device__ __forceinline__ double i32_to_f64(uint32_t a) {
  return __hiloint2double(0x43380000, (int)(a ^ 0x80000000u)) - 6755401588539392.0;
}

// Instruction descriptor: S8 x S8 -> S32, both K-major, M = 128, N = NT(S).
__host__ __device__ constexpr uint32_t instr_desc_i8(int nt) {
  return (2u << 4)                      // D format S32
         | (1u << 7) | (1u << 10)       // A, B format S8
         | ((uint32_t)(nt >> 3) << 17)  // N
         | ((uint32_t)(BM >> 4) << 24); // M
}
// A-operand collector use of one MMA: the MMAs of one A slice (pairs (s, t) for
// t = 0..S-1-s) run back to back, so the first fills the collector buffer from
// shared memory, the middle ones use it and the last releases it; an A slice with
// a single MMA reads shared memory as usual.  Each reuse saves one A tile read
// (128 x 32 bytes) from shared memory, whose bandwidth bounds this kernel.
enum CollectorOp { kCollNone = 0, kCollFill = 1, kCollUse = 2, kCollLast = 3 };
template <int kOp>
__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
#define TRHEPD_MMA_I8(Q)                                                                   \
  asm volatile("{\n\t.reg .pred p;\n\t"                                                  \
               "setp.ne.b32 p, %4, 0;\n\t"                                                \
               "tcgen05.mma.cta_group::1.kind::i8" Q " [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem), \
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)                          \
               : "memory")
  if constexpr (kOp == kCollFill) TRHEPD_MMA_I8(".collector::a::fill");
  else if constexpr (kOp == kCollUse) TRHEPD_MMA_I8(".collector::a::use");
  else if constexpr (kOp == kCollLast) TRHEPD_MMA_I8(".collector::a::lastuse");
  else TRHEPD_MMA_I8("");
#undef TRHEPD_MMA_I8
}

// Balanced base-256 digits of X = rint(x * scale), scale = 2^(7 - e + 8(S-1)),
// most significant first.  |X| < 2^(7 + 8(S-1)): 32-bit arithmetic for S <= 4,
// 64-bit for S = 5, 6 (|X| < 2^47, exact in double before the rounding).
template <int S>
__device__ __forceinline__ void digits_i8(double x, double scale, int* d) {
  static_assert(S <= 6, "at most six digits");
  if constexpr (S <= 4) {
    int X = __double2int_rn(x * scale);
#pragma unroll
    for (int s = S - 1; s >= 1; --s) {
      const int lo = ((X + 128) & 255) - 128;
      d[s] = lo;
      X = (X - lo) >> 8;
    }
    d[0] = X;
  } else {
    long long X = __double2ll_rn(x * scale);
#pragma unroll
    for (int s = S - 1; s >= 1; --s) {
      const int lo = (int)((X + 128) & 255) - 128;
      d[s] = lo;
      X = (X - lo) >> 8;
    }
    d[0] = (int)X;
  }
}
__device__ __forceinline__ double digit_scale(int e, int S) {
  return pow2(7 - e + 8 * (S - 1));
}
__device__ __forceinline__ uint32_t pack4(int a, int b, int c, int d) {
  return (uint32_t)(a & 255) | ((uint32_t)(b & 255) << 8) | ((uint32_t)(c & 255) << 16) |
         ((uint32_t)(d & 255) << 24);
}
__device__ __forceinline__ uint16_t pack2(int a, int b) {
  return (uint16_t)((a & 255) | ((b & 255) << 8));
}

// One warp per stacked row: exponent of the off-diagonal row maximum, then the S
// digit slices of the row, (Re, Im) interleaved; each lane writes two complex k.
template <int S, int NPL>
__global__ void __launch_bounds__(256) k_slice_rows_i8(const cd* __restrict__ Q, int rows, int n,
                                                       int ld, int kc, uint16_t* __restrict__ A,
                                                       int* __restrict__ erow) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= rows) return;
  const int r = warp, i = r % n;
  const cd* q = Q + (size_t)r * ld;
  // one pass over the row: lane holds complex k = lane + 32 j (k < kc, zero past n
  // and on the diagonal), the row maximum, then the digits from registers
  cd v[NPL];
  double m = 0.0;
#pragma unroll
  for (int j = 0; j < NPL; ++j) {
    const int k = lane + 32 * j;
    v[j] = (k < n && k != i) ? q[k] : cd{0.0, 0.0};
    m = fmax(m, fmax(fabs(v[j].x), fabs(v[j].y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  int e = 0;
  if (m > 0.0) frexp(m * kDigitHeadroom, &e);
  if (lane == 0) erow[r] = e;
  const double sc = digit_scale(e, S);
#pragma unroll
  for (int j = 0; j < NPL; ++j) {
    const int k = lane + 32 * j;
    if (k < kc) {
      int a[S], b[S];
      digits_i8<S>(v[j].x, sc, a);
      digits_i8<S>(v[j].y, sc, b);
#pragma unroll
      for (int s = 0; s < S; ++s) A[((size_t)s * rows + r) * kc + k] = pack2(a[s], b[s]);
    }
  }
}

// One block per column j of Voff: the column exponent (maximum times the
// headroom), then the B^T digit slices: row 2j (Re-out) = [Vr(k,j), -Vi(k,j)]_k,
// row 2j+1 (Im-out) = [Vi, Vr]_k; -Vi gets its own digits (negating digits could
// leave 128).
template <int S>
__global__ void __launch_bounds__(128) k_slice_cols_i8(const cd* __restrict__ V, int n, int ld,
                                                        int kc, int nrows, int* __restrict__ fcol,
                                                        uint16_t* __restrict__ B,
                                                        long long vstride, int fstride) {
  __shared__ double red[4];
  const int j = blockIdx.x, tid = threadIdx.x;
  V += (size_t)blockIdx.y * vstride;  // problem blockIdx.y of a stacked group
  fcol += (size_t)blockIdx.y * fstride;
  B += (size_t)blockIdx.y * S * nrows * kc;
  double m = 0.0;
  for (int k = tid; k < n; k += 128) {
    const cd v = V[(size_t)k * ld + j];
    m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((tid & 31) == 0) red[tid >> 5] = m;
  __syncthreads();
  m = fmax(fmax(red[0], red[1]), fmax(red[2], red[3]));
  int e = 0;
  if (m > 0.0) frexp(m * kDigitHeadroom, &e);
  if (tid == 0) fcol[j] = e;
  const double sc = digit_scale(e, S);
  for (int k = tid; k < kc; k += 128) {
    const cd v = (k < n) ? V[(size_t)k * ld + j] : cd{0.0, 0.0};
    int dr[S], di[S], dn[S];
    digits_i8<S>(v.x, sc, dr);
    digits_i8<S>(v.y, sc, di);
    digits_i8<S>(-v.y, sc, dn);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      B[((size_t)s * nrows + 2 * j) * kc + k] = pack2(dr[s], dn[s]);
      B[((size_t)s * nrows + 2 * j + 1) * kc + k] = pack2(di[s], dr[s]);
    }
  }
}

// Called once per CTA when it has claimed its last tile: the last CTA of the launch
// re-arms the counter pair (next tile, finished CTAs) for the next launch on the
// stream (kernel boundaries order the reset before that launch's claims).
__device__ __forceinline__ void tile_counter_done(int* counter, unsigned ctas) {
  __threadfence();
  if (atomicAdd(&counter[1], 1) == (int)ctas - 1) {
    counter[0] = 0;
    counter[1] = 0;
    __threadfence();
  }
}

#ifndef TRHEPD_COLLECT_A
#define TRHEPD_COLLECT_A 1
#endif
constexpr bool kCollectA = TRHEPD_COLLECT_A != 0;  // A-slice reuse through the MMA collector

// Persistent INT8 stage product: one CTA per SM (or fewer) takes tiles from a
// per-launch counter; warp 0 claims them and issues TMA, warp 1 the MMAs of every slice pair (s, t) with s + t < S into
// accumulator level s + t, warps 2-3 idle; eight epilogue warps (two per TMEM lane
// quadrant, one per column half) drain a finished tile into registers, give the
// TMEM back at once (the next tile's MMAs start) and perform the FP64 RKN update
// from registers.  Tile: 128 stacked rows x NT(S) real columns; S levels x NT(S)
// TMEM columns.  setmaxnreg splits the registers (control 40, epilogue 232).
template <int S>
__global__ void __launch_bounds__(P_THREADS, 1)
    k_split_gemm_i8(const __grid_constant__ CUtensorMap tmA,
                    const __grid_constant__ CUtensorMap tmB, EpiArgs ep, int nkb, int tiles_n,
                    int tiles, int dpitch) {
  constexpr int NTS = i8::nt_for(S);          // real columns per tile
  constexpr int NCS = NTS / 2;                // complex columns per tile
  constexpr int G = NCS / 8;                  // 4-column groups per epilogue warp
  constexpr int STEPS = 2 * G;                // update steps (g, h) per tile
  constexpr int STAGES = i8::STAGES;
  constexpr int RING = i8::ring_slots(S);
  constexpr int AHEAD = RING - 1;             // ring steps in flight
  constexpr int VA = i8::v_ahead(S);          // stage-matrix steps in flight
  static_assert(S * NTS <= TMEM_COLS, "INT8 levels exceed the tensor memory");
  static_assert(NCS % 8 == 0 && NTS % 16 == 0, "tile width");
  constexpr int TQ = 4;                       // tile-index queue slots
  if (*(volatile unsigned*)ep.status & kStatusTimeout) {
    if (threadIdx.x == 0) tile_counter_done(ep.tile_counter, gridDim.x);
    return;
  }
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], tfull, tempty, drain_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh, issued_sh, consumed_sh;
  // Tiles are claimed dynamically from a per-launch counter by the TMA warp and
  // handed to the MMA and epilogue warps through a queue of TQ slots (-1: no more):
  // a CTA that starts late (its SM held by another kernel) takes what is left.
  __shared__ int tq[TQ];
  __shared__ __align__(8) uint64_t tq_full[TQ], tq_empty[TQ];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t sbytes = i8::stage_bytes(S);
  constexpr int BSL = i8::b_slice_bytes(S);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&tfull, 1);
    mbar_init(&tempty, P_EPI_WARPS);
    mbar_init(&drain_bar, 1);
    for (int q = 0; q < TQ; ++q) {
      mbar_init(&tq_full[q], 1);
      mbar_init(&tq_empty[q], 1 + P_EPI_WARPS);  // the MMA thread and every epilogue warp
    }
    abort_sh = 0;
    issued_sh = 0;
    consumed_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(P_REG_CTRL));
    if (warp == 0) {
      // ---------------- TMA producer
      if (lane == 0) {
        int g = 0;
        bool stop = false;
        for (int it = 0; !stop; ++it) {
          // claim the next tile and publish it in queue slot it % TQ
          const int qs = it % TQ;
          if (it >= TQ && !mbar_wait(&tq_empty[qs], ((it / TQ) - 1) & 1)) {
            atomicOr(ep.status, kStatusTimeout);
            abort_sh = 1;
            break;
          }
          int tile = ld_volatile(&abort_sh) ? tiles : atomicAdd(ep.tile_counter, 1);
          if (tile >= tiles) tile = -1;
          tq[qs] = tile;
          mbar_arrive(&tq_full[qs]);
          if (tile < 0) break;
          const int rt = tile / tiles_n, pb = rt / ep.tpp;
          const int m0 = pb * ep.rows_b + (rt - pb * ep.tpp) * BM, n0 = (tile % tiles_n) * NTS;
          for (int kb = 0; kb < nkb; ++kb, ++g) {
            const int st = g % STAGES, round = g / STAGES;
            if (round > 0 && !mbar_wait(&empty_bar[st], (round - 1) & 1)) {
              atomicOr(ep.status, kStatusTimeout);
              abort_sh = 1;
              stop = true;
              break;
            }
            if (ld_volatile(&abort_sh)) {
              stop = true;
              break;
            }
            unsigned char* sa = smem + st * sbytes;
            unsigned char* sb = sa + S * i8::A_SLICE_BYTES;
            mbar_expect_tx(&full_bar[st], (uint32_t)sbytes);
#pragma unroll
            for (int s = 0; s < S; ++s) {
              tma_load_3d(&tmA, &full_bar[st], sa + s * i8::A_SLICE_BYTES, kb * i8::BK, m0, s);
              tma_load_3d(&tmB, &full_bar[st], sb + s * BSL, kb * i8::BK, n0, pb * S + s);
            }
          }
        }
        issued_sh = g;
      }
    } else if (warp == 1) {
      // ---------------- MMA issuer
      if (lane == 0) {
        const uint32_t idesc = instr_desc_i8(NTS);
        int g = 0, it = 0;
        bool stop = false;
        for (;; ++it) {
          const int qs = it % TQ;
          if (!mbar_wait(&tq_full[qs], (it / TQ) & 1)) {
            atomicOr(ep.status, kStatusTimeout);
            abort_sh = 1;
            break;
          }
          const int tile = tq[qs];
          mbar_arrive(&tq_empty[qs]);
          if (tile < 0) break;
          if (it > 0 && !mbar_wait(&tempty, (it - 1) & 1)) {
            atomicOr(ep.status, kStatusTimeout);
            abort_sh = 1;
            break;
          }
          tc_fence_after();
          bool started[S];
#pragma unroll
          for (int L = 0; L < S; ++L) started[L] = false;
          for (int kb = 0; kb < nkb; ++kb, ++g) {
            const int st = g % STAGES, round = g / STAGES;
            if (!mbar_wait(&full_bar[st], round & 1)) {
              atomicOr(ep.status, kStatusTimeout);
              abort_sh = 1;
              stop = true;
              break;
            }
            tc_fence_after();
            const uint32_t sa = smem_u32(smem + st * sbytes);
            const uint32_t sb = sa + S * i8::A_SLICE_BYTES;
#pragma unroll
            for (int kk = 0; kk < i8::BK / 32; ++kk) {
#pragma unroll
              for (int s = 0; s < S; ++s) {
#pragma unroll
                for (int t = 0; t < S - s; ++t) {
                  const int L = s + t;
                  const uint64_t ad = sw64_desc(sa + s * i8::A_SLICE_BYTES + kk * 32);
                  const uint64_t bd = sw64_desc(sb + t * BSL + kk * 32);
                  const uint32_t acc = started[L] ? 1u : 0u;
                  if (!kCollectA || S - s == 1) tc_mma_i8<kCollNone>(tmem + L * NTS, ad, bd, idesc, acc);
                  else if (t == 0) tc_mma_i8<kCollFill>(tmem + L * NTS, ad, bd, idesc, acc);
                  else if (t == S - s - 1) tc_mma_i8<kCollLast>(tmem + L * NTS, ad, bd, idesc, acc);
                  else tc_mma_i8<kCollUse>(tmem + L * NTS, ad, bd, idesc, acc);
                  started[L] = true;
                }
              }
            }
            tc_commit(&empty_bar[st]);
          }
          if (stop) break;
          tc_commit(&tfull);
        }
        consumed_sh = g;
        tc_commit(&drain_bar);
        if (!mbar_wait(&drain_bar, 0)) atomicOr(ep.status, kStatusTimeout);
      }
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(P_REG_EPI));
    // ---------------- epilogue warps 4..11
    // Warp w (q4 = w & 3: TMEM lane quadrant, rows q4*32..+31 of the tile; half:
    // complex columns half*NCS/2..+NCS/2-1) holds per lane rows t1, t1 + 8 of its
    // 16-row blocks h = 0, 1 and complex column t0 of its 4-column groups g < G.
    // Update step ls = 2g + h, STEPS per tile.
    const int q4 = warp & 3;
    const int ew = warp - 4;
    const int half = ew >> 2;
    const int t0 = lane & 3, t1 = lane >> 2;
    unsigned char* dtab_base = smem + STAGES * sbytes;
    double2* ring = reinterpret_cast<double2*>(dtab_base + 2 * i8::kDTabBytes) + ew * 32 + lane;
    const uint32_t ring_s = smem_u32(ring);
    constexpr int kItem = P_EPI_WARPS * 32;               // double2 entries between items
    constexpr uint32_t kItemBytes = kItem * 16;
    // Row block of a tile for this warp: first row, end of its problem's rows,
    // first complex column (rend = 0 past the last tile: nothing to load).
    struct Geo {
      int m0, rend, jh;
    };
    auto geometry = [&](int tile) {
      Geo Gt{0, 0, 0};
      if (tile >= 0 && tile < tiles) {
        const int rt = tile / tiles_n, pb = rt / ep.tpp;
        Gt.m0 = pb * ep.rows_b + (rt - pb * ep.tpp) * BM + q4 * 32;
        Gt.rend = min(ep.rows, (pb + 1) * ep.rows_b);
        Gt.jh = (tile % tiles_n) * NCS + half * (NCS / 2);
      }
      return Gt;
    };
    // cp.async the Q and P entries of step ls of the tile with geometry Gt into ring
    // slot `slot` (one commit group per step, empty outside the matrix)
    auto issue = [&](const Geo& Gt, int ls, int slot) {
      const int g = ls >> 1, h = ls & 1;
      const int j = Gt.jh + 4 * g + t0;
      const uint32_t sa = ring_s + (uint32_t)slot * i8::kRingItems * kItemBytes;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int r = Gt.m0 + 16 * h + 8 * u + t1;
        if (r < Gt.rend && j < ep.n) {
          const size_t o = (size_t)r * ep.ld + j;
          cp_async_16(sa + u * kItemBytes, ep.Q + o);
          cp_async_16(sa + (2 + u) * kItemBytes, ep.P + o);
        }
      }
      cp_async_commit();
    };
    int slot_rd = 0, slot_wr = 0;
    auto next_slot = [](int s) { return s + 1 == RING ? 0 : s + 1; };
    // the first tile of this CTA (-1: none); each tile has more than AHEAD steps
    bool qok = mbar_wait(&tq_full[0], 0);
    int tile = qok ? tq[0] : -1;
    {
      const Geo G0 = geometry(tile);
#pragma unroll
      for (int q = 0; q < AHEAD; ++q) {
        issue(G0, q, slot_wr);
        slot_wr = next_slot(slot_wr);
      }
    }
    if (epi_any(!qok)) {
      if (!qok) atomicOr(ep.status, kStatusTimeout);
      abort_sh = 1;
      tile = -1;
    }
    int it = 0;
    for (; tile >= 0; ++it) {
      const int rt = tile / tiles_n, pb = rt / ep.tpp;
      const int m0 = pb * ep.rows_b + (rt - pb * ep.tpp) * BM + q4 * 32;
      const int rend = min(ep.rows, (pb + 1) * ep.rows_b);  // this problem's rows end here
      const int j0 = (tile % tiles_n) * NCS;                 // first column of the tile
      const int jh = j0 + half * (NCS / 2);
      const cd* Vb = ep.V + (size_t)pb * ep.vstride;
      const int* fcb = ep.fcol + (size_t)pb * ep.fstride;
      const cd vd = Vb[(size_t)ep.kpad * ep.ld];
      // the next tile of this CTA, published by the TMA warp before it loads that
      // tile's operands (so before this tile's MMAs finish)
      const int qn = (it + 1) % TQ;
      const bool nok = mbar_wait(&tq_full[qn], ((it + 1) / TQ) & 1);
      const int tile_next = nok ? tq[qn] : -1;
      const Geo Gc{m0, rend, jh}, Gn = geometry(tile_next);
      // D table of this tile: angles a0.. of its rows, columns j0 .. j0 + dpitch - 1
      const int tm0 = m0 - q4 * 32;
      const int a0 = tm0 / ep.n;
      const int na = (min(tm0 + BM, rend) - 1) / ep.n - a0 + 1;
      cd* dtab = reinterpret_cast<cd*>(dtab_base + (it & 1) * i8::kDTabBytes);
      for (int e = (warp - 4) * 32 + lane; e < na * dpitch; e += P_EPI_WARPS * 32) {
        const int a = e / dpitch, jl = e - a * dpitch;
        const int j = j0 + jl;
        dtab[e] = (j < ep.n) ? ep.D[(size_t)(a0 + a) * ep.ld + j] + vd : cd{0.0, 0.0};
      }
      int er[2][2], ra[2][2], ri[2][2];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int r = m0 + 16 * h + 8 * u + t1;
          er[h][u] = 0;
          ra[h][u] = 0;
          ri[h][u] = 0;
          if (r < rend) {
            er[h][u] = ep.erow[r];
            ra[h][u] = r / ep.n;
            ri[h][u] = r - ra[h][u] * ep.n;
          }
        }
      int fc[G];
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const int j = jh + 4 * g + t0;
        fc[g] = (j < ep.n) ? fcb[j] : 0;
      }
      cd qd[2][2];  // diagonal of each of this lane's rows (read while the MMAs run)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int r = m0 + 16 * h + 8 * u + t1;
          qd[h][u] = (r < rend) ? ep.Q[(size_t)r * ep.ld + ri[h][u]] : cd{0.0, 0.0};
        }
      // the stage matrix entries of the first VA steps
      cd vq[VA][2];
#pragma unroll
      for (int ls = 0; ls < VA; ++ls) {
        const int g = ls >> 1, h = ls & 1, j = jh + 4 * g + t0;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int r = m0 + 16 * h + 8 * u + t1;
          vq[ls][u] = (r < rend && j < ep.n) ? Vb[(size_t)ri[h][u] * ep.ld + j] : cd{0.0, 0.0};
        }
      }
      const bool ok = nok && mbar_wait(&tfull, it & 1);
      // also the barrier after which every epilogue warp sees this tile's D table
      if (epi_any(!ok)) {
        if (!ok) atomicOr(ep.status, kStatusTimeout);
        abort_sh = 1;
        break;
      }
      tc_fence_after();
      // drain: each level's INT32 sums as exact doubles, combined by Horner in
      // powers of 2^-8, then scaled by 2^(e_r + f_j - 14)
      cd vals[G][2][2];
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t taddr = tmem + ((uint32_t)(q4 * 32 + 16 * h) << 16) +
                                 (uint32_t)(2 * (half * (NCS / 2) + 4 * g));
          uint32_t a[S][4];
#pragma unroll
          for (int L = 0; L < S; ++L) tmem_ld_16x256(taddr + L * NTS, a[L]);
          tmem_wait_ld();
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            double re = i32_to_f64(a[S - 1][2 * u]), im = i32_to_f64(a[S - 1][2 * u + 1]);
#pragma unroll
            for (int L = S - 2; L >= 0; --L) {
              re = fma(re, 0.00390625, i32_to_f64(a[L][2 * u]));
              im = fma(im, 0.00390625, i32_to_f64(a[L][2 * u + 1]));
            }
            const double sc = pow2(er[h][u] + fc[g] - 14);
            vals[g][h][u] = cd{re * sc, im * sc};
          }
        }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty);
#pragma unroll
      for (int ls = 0; ls < STEPS; ++ls) {
        const int g = ls >> 1, h = ls & 1;
        const int j = jh + 4 * g + t0;
        cp_async_wait<AHEAD - 1>();  // this step's group has landed
        const double2* sl = ring + slot_rd * (i8::kRingItems * kItem);
        cd qv[2], pv[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const double2 x = sl[u * kItem], y = sl[(2 + u) * kItem];
          qv[u] = cd{x.x, x.y};
          pv[u] = cd{y.x, y.y};
        }
        slot_rd = next_slot(slot_rd);
        // the slot refilled now is the one read (and used) by the previous step
        if (ls + AHEAD < STEPS)
          issue(Gc, ls + AHEAD, slot_wr);
        else
          issue(Gn, ls + AHEAD - STEPS, slot_wr);
        slot_wr = next_slot(slot_wr);
        const cd vv[2] = {vq[ls % VA][0], vq[ls % VA][1]};
        if (ls + VA < STEPS) {  // the stage-matrix entries VA steps ahead
          const int g2 = (ls + VA) >> 1, h2 = (ls + VA) & 1, j2 = jh + 4 * g2 + t0;
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int r = m0 + 16 * h2 + 8 * u + t1;
            if (r < rend && j2 < ep.n) vq[ls % VA][u] = Vb[(size_t)ri[h2][u] * ep.ld + j2];
          }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int r = m0 + 16 * h + 8 * u + t1;
          if (r < rend && j < ep.n) {
            const size_t ro = (size_t)r * ep.ld;
            const cd dv = dtab[(ra[h][u] - a0) * dpitch + (j - j0)];
            const cd acc = vals[g][h][u] + qd[h][u] * vv[u] + qv[u] * dv;
            const cd p = pv[u] + ep.cb * acc;
            ep.P[ro + j] = p;
            ep.Qo[ro + j] = qv[u] + ep.ca * p;
          }
        }
      }
      // queue slot of this tile no longer read by this warp (the next one is kept
      // until the end of the next tile)
      __syncwarp();
      if (lane == 0) mbar_arrive(&tq_empty[it % TQ]);
      tile = tile_next;
    }
    cp_async_wait<0>();
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int g = consumed_sh; g < issued_sh; ++g)
      if (!mbar_wait(&full_bar[g % STAGES], (g / STAGES) & 1)) break;
  }
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
  if (threadIdx.x == 0) tile_counter_done(ep.tile_counter, gridDim.x);
}

}  // namespace split

// Row slicing with the row held in registers: complex entries per lane NPL >=
// ceil(kc / 32), the smallest instantiated (kc <= 832).
template <int S>
static void slice_rows_i8(const cd* Q, int rows, int n, int ld, int kc, uint16_t* A, int* erow,
                          cudaStream_t st) {
  const int blocks = ceil_div(rows, 8), npl = ceil_div(kc, 32);
  if (npl <= 2) split::k_slice_rows_i8<S, 2><<<blocks, 256, 0, st>>>(Q, rows, n, ld, kc, A, erow);
  else if (npl <= 4) split::k_slice_rows_i8<S, 4><<<blocks, 256, 0, st>>>(Q, rows, n, ld, kc, A, erow);
  else if (npl <= 8) split::k_slice_rows_i8<S, 8><<<blocks, 256, 0, st>>>(Q, rows, n, ld, kc, A, erow);
  else if (npl <= 12) split::k_slice_rows_i8<S, 12><<<blocks, 256, 0, st>>>(Q, rows, n, ld, kc, A, erow);
  else if (npl <= 17) split::k_slice_rows_i8<S, 17><<<blocks, 256, 0, st>>>(Q, rows, n, ld, kc, A, erow);
  else split::k_slice_rows_i8<S, 26><<<blocks, 256, 0, st>>>(Q, rows, n, ld, kc, A, erow);
}

// ============================================================ host side
namespace {

struct Carve {
  __nv_bfloat162* A;
  __nv_bfloat162* B;
  int* erow;
  int* fcol;
  int* counter;  // the INT8 kernel's tile counter pair (zeroed with the workspace)
  int rows, kc, npad, nrows;
};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Workspace layout: A slices, B^T slices (`cbytes` bytes per complex entry: 4 for
// BF16 pairs, 2 for INT8 pairs; one set per problem of a stacked group), row and
// column exponents.
Carve carve(void* base, int nang, int n, int S, int cbytes = 4, int nprob = 1,
            int nc = split::NC) {
  Carve c;
  c.rows = nang * n;
  c.kc = round_up(n, 16);                 // complex k (= ld of the state)
  c.npad = round_up(n, nc);               // complex columns of the tiles
  c.nrows = 2 * c.npad;
  char* p = reinterpret_cast<char*>(base);
  size_t o = 0;
  c.A = reinterpret_cast<__nv_bfloat162*>(p + o);
  o = align256(o + (size_t)S * c.rows * c.kc * cbytes);
  c.B = reinterpret_cast<__nv_bfloat162*>(p + o);
  o = align256(o + (size_t)nprob * S * c.nrows * c.kc * cbytes);
  c.erow = reinterpret_cast<int*>(p + o);
  o = align256(o + (size_t)c.rows * sizeof(int));
  c.fcol = reinterpret_cast<int*>(p + o);
  o = align256(o + (size_t)nprob * c.npad * sizeof(int));
  c.counter = reinterpret_cast<int*>(p + o);  // in the 256 bytes split_workspace_bytes adds
  return c;
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      throw std::runtime_error("cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

// 3-D map over [S][rows][kr] elements of `esize` bytes (BF16 or INT8) with a
// (64 bytes x box_rows x 1) box and 64-byte swizzle; out-of-range boxes read zeros.
CUtensorMap make_map(void* base, int kr, int rows, int S, int esize = 2, int box_rows = split::BM) {
  CUtensorMap m;
  cuuint64_t dims[3] = {(cuuint64_t)kr, (cuuint64_t)rows, (cuuint64_t)S};
  cuuint64_t strides[2] = {(cuuint64_t)kr * esize, (cuuint64_t)kr * esize * rows};
  cuuint32_t box[3] = {(cuuint32_t)(64 / esize), (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType dt =
      (esize == 2) ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  CUresult r = encoder()(&m, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

int current_device() {
  int dev = 0;
  cudaGetDevice(&dev);
  return dev;
}

int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

// CTAs of a persistent kernel: one per SM, or fewer when the context caps them (a
// serving slot leaving SMs to concurrent requests of other slots).
// CTAs of a persistent split kernel: one per SM, at most max_ctas (> 0), or one
// per tile (max_ctas = -1: each CTA takes about one tile and exits, so the block
// scheduler can start higher-priority work of other streams between tiles).
int persistent_grid(const SplitWorkspace& w) {
  const int sms = sm_count();
  if (w.max_ctas < 0) return 1 << 30;
  return w.max_ctas > 0 ? std::min(sms, w.max_ctas) : sms;
}

template <int S>
void run_split(const SplitWorkspace& w, const cd* Q, cd* P, cd* Qo, const cd* V, const cd* D,
               int nang, int n, int ld, double cb, double ca, int variant, const cudaEvent_t* ev,
               cudaStream_t st) {
  Carve c = carve(w.base, nang, n, S);
  const int kr = 2 * c.kc;
  // slices of the shared potential matrix (one set for every angle)
  split::k_col_exponents<<<ceil_div(n, 32), 256, 0, st>>>(V, n, ld, 1.0, c.fcol);
  {
    dim3 grid(ceil_div(c.kc, 128), n);
    split::k_slice_cols<S><<<grid, 128, 0, st>>>(V, n, ld, c.kc, c.nrows, c.fcol, c.B);
  }
  // slices of the stacked states
  split::k_slice_rows<S><<<ceil_div(c.rows, 8), 256, 0, st>>>(Q, c.rows, n, ld, kr, c.A, c.erow);
  CUtensorMap ta = make_map(c.A, kr, c.rows, S);
  CUtensorMap tb = make_map(c.B, kr, c.nrows, S);
  split::EpiArgs ep{Q, P, Qo, V, D, c.erow, c.fcol, w.status, c.rows, n, ld, c.kc, S, cb, ca};
  const int tiles_n = c.nrows / split::NT, tiles_m = ceil_div(c.rows, split::BM);
  if (variant == kSplitPersistent) {
    const size_t smem = split::psmem_bytes(S);
    static SmemOptIn attr;
    if (!attr.bytes_on(current_device())) {
      // setmaxnreg redistributes the registers the block was launched with: the
      // kernel must have been built with the count the split assumes
      cudaFuncAttributes fa{};
      if (cudaFuncGetAttributes(&fa, split::k_split_gemm_p<S>) != cudaSuccess ||
          fa.numRegs < split::P_REG_LAUNCH)
        throw std::runtime_error("persistent split kernel built with " +
                                 std::to_string(fa.numRegs) + " registers per thread, needs " +
                                 std::to_string(split::P_REG_LAUNCH));
    }
    attr.ensure((const void*)split::k_split_gemm_p<S>, smem);
    const int tiles = tiles_n * tiles_m;
    const int grid = std::min(tiles, persistent_grid(w));
    if (ev) cudaEventRecord(ev[0], st);
    split::k_split_gemm_p<S><<<grid, split::P_THREADS, smem, st>>>(ta, tb, ep, kr / split::BK,
                                                                   tiles_n, tiles);
    if (ev) cudaEventRecord(ev[1], st);
  } else {
    const size_t smem = split::smem_bytes(S);
    static SmemOptIn attr;
    attr.ensure((const void*)split::k_split_gemm<S>, smem);
    dim3 grid(tiles_n, tiles_m);
    if (ev) cudaEventRecord(ev[0], st);
    split::k_split_gemm<S><<<grid, split::THREADS, smem, st>>>(ta, tb, ep, kr / split::BK);
    if (ev) cudaEventRecord(ev[1], st);
  }
}

template <int S>
void run_split_i8(const SplitWorkspace& w, const cd* Q, cd* P, cd* Qo, const cd* V, const cd* D,
                  int nang, int n, int ld, double cb, double ca, const cudaEvent_t* ev,
                  StackedRows sr, cudaStream_t st) {
  constexpr int NTS = split::i8::nt_for(S), NCS = NTS / 2;
  const int rows = nang * n;
  if (sr.rows_b <= 0) sr = StackedRows{rows, 0};
  const int nprob = ceil_div(rows, sr.rows_b);
  Carve c = carve(w.base, nang, n, S, 2, nprob, NCS);
  const int kr = 2 * c.kc;
  if (kr > 16384) throw std::invalid_argument("INT8 split form: k beyond the exact INT32 range");
  uint16_t* B = reinterpret_cast<uint16_t*>(c.B);
  split::k_slice_cols_i8<S><<<dim3(n, nprob), 128, 0, st>>>(V, n, ld, c.kc, c.nrows, c.fcol, B,
                                                            sr.vstride, c.npad);
  slice_rows_i8<S>(Q, c.rows, n, ld, c.kc, reinterpret_cast<uint16_t*>(c.A), c.erow, st);
  CUtensorMap ta = make_map(c.A, kr, c.rows, S, 1);
  CUtensorMap tb = make_map(c.B, kr, c.nrows, S * nprob, 1, NTS);
  split::EpiArgs ep{Q, P, Qo, V, D, c.erow, c.fcol, w.status, c.rows, n, ld, c.kc, S, cb, ca};
  const int tpp = ceil_div(sr.rows_b, split::BM);
  ep.rows_b = sr.rows_b;
  ep.vstride = sr.vstride;
  ep.fstride = c.npad;
  ep.tpp = tpp;
  ep.tile_counter = c.counter;
  // the epilogue's per-tile table of D: the angles of 128 rows x min(NC, n) columns
  const int dpitch = std::min(NCS, n);
  if ((size_t)((split::BM - 1) / n + 2) * dpitch * sizeof(cd) > (size_t)split::i8::kDTabBytes)
    throw std::invalid_argument("INT8 split form: diagonal table exceeds its shared memory");
  const int tiles_n = c.nrows / NTS, tiles_m = nprob * tpp;
  const size_t smem = split::i8::smem_bytes(S);
  static SmemOptIn attr;
  if (!attr.bytes_on(current_device())) {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, split::k_split_gemm_i8<S>) != cudaSuccess ||
        fa.numRegs < split::P_REG_LAUNCH)
      throw std::runtime_error("INT8 split kernel built with " + std::to_string(fa.numRegs) +
                               " registers per thread, needs " +
                               std::to_string(split::P_REG_LAUNCH));
  }
  attr.ensure((const void*)split::k_split_gemm_i8<S>, smem);
  const int tiles = tiles_n * tiles_m;
  const int grid = std::min(tiles, persistent_grid(w));
  if (ev) cudaEventRecord(ev[0], st);
  split::k_split_gemm_i8<S><<<grid, split::P_THREADS, smem, st>>>(
      ta, tb, ep, ceil_div(kr, split::i8::BK), tiles_n, tiles, dpitch);
  if (ev) cudaEventRecord(ev[1], st);
}

}  // namespace

size_t split_workspace_bytes(int nang, int n, int slices, int nprob) {
  // large enough for every tile width (BF16: 64 complex columns; INT8: 64, 48, 40)
  size_t b = 0;
  for (int nc : {split::NC, split::i8::nc_for(5), split::i8::nc_for(6)}) {
    Carve c = carve(nullptr, nang, n, slices, 4, nprob, nc);
    b = std::max(b, reinterpret_cast<size_t>(c.fcol) +
                        align256((size_t)nprob * c.npad * sizeof(int)) + 256);
  }
  return b;
}

SplitWorkspace split_workspace_carve(void* base, int nang, int n, int slices, unsigned* status,
                                     cudaStream_t st, int nprob) {
  SplitWorkspace w;
  w.base = base;
  w.nang = nang;
  w.n = n;
  w.slices = slices;
  w.status = status;
  // padded rows of the slice buffers are never written by the slicing kernels
  cudaMemsetAsync(base, 0, split_workspace_bytes(nang, n, slices, nprob), st);
  return w;
}

int split_stage(const SplitWorkspace& w, const cd* Q, cd* P, cd* Qo, const cd* V, const cd* D,
                int nang, int n, int ld, double cb, double ca, int slices, int variant,
                const cudaEvent_t* ev, cudaStream_t st, StackedRows sr) {
  if (variant == kSplitInt8) {
    switch (slices) {
      case 3:
        run_split_i8<3>(w, Q, P, Qo, V, D, nang, n, ld, cb, ca, ev, sr, st);
        break;
      case 4:
        run_split_i8<4>(w, Q, P, Qo, V, D, nang, n, ld, cb, ca, ev, sr, st);
        break;
      case 5:
        run_split_i8<5>(w, Q, P, Qo, V, D, nang, n, ld, cb, ca, ev, sr, st);
        break;
      case 6:
        run_split_i8<6>(w, Q, P, Qo, V, D, nang, n, ld, cb, ca, ev, sr, st);
        break;
      default:
        throw std::invalid_argument("INT8 split slices must be 3 to 6");
    }
    return 4;
  }
  if (variant != kSplitPersistent && variant != kSplitPerTile)
    throw std::invalid_argument("unknown split kernel variant");
  if (sr.rows_b > 0 && sr.rows_b < nang * n)
    throw std::invalid_argument("stacked problems run the INT8 or FP64 form only");
  switch (slices) {
    case 3:
      run_split<3>(w, Q, P, Qo, V, D, nang, n, ld, cb, ca, variant, ev, st);
      break;
    case 4:
      run_split<4>(w, Q, P, Qo, V, D, nang, n, ld, cb, ca, variant, ev, st);
      break;
    case 5:
      run_split<5>(w, Q, P, Qo, V, D, nang, n, ld, cb, ca, variant, ev, st);
      break;
    default:
      throw std::invalid_argument("split slices must be 3, 4 or 5");
  }
  return 4;
}

}  // namespace trhepd
