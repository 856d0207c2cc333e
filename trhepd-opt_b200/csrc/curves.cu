// Rocking-curve epilogues on the device: per-curve error of a split-precision
// solve against the FP64 form, and the curve-comparison metric of the
// reference's regression scripts (test/test23/compare.py:50-67).  Both reduce
// the (angles x beams) intensities of a resident problem to a few numbers per
// angle, so only those cross to the host.
#include <cuda_runtime.h>

#include "curves.h"

namespace trhepd {

namespace {

// Block-wide maximum / sum of one value per thread (blockDim.x = 256).
template <bool kMax>
__device__ double block_reduce(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = kMax ? fmax(v, w) : v + w;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;  // every value is >= 0
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = kMax ? fmax(v, w) : v + w;
    }
    if (lane == 0) sh[0] = v;
  }
  __syncthreads();
  return sh[0];
}

// One block per curve (angle): out[3a] = max over spots of |got - ref| / |ref|
// (a spot with ref = 0 counts 0 when got = 0 too, else infinity), out[3a+1] =
// max |got - ref| / max |ref| of the curve, out[3a+2] = max |ref|.
__global__ void __launch_bounds__(256) k_curve_errors(const double* __restrict__ got,
                                                      const double* __restrict__ ref, int nb,
                                                      double* __restrict__ out) {
  __shared__ double sh[32];
  const int a = blockIdx.x;
  const double* g = got + (size_t)a * nb;
  const double* r = ref + (size_t)a * nb;
  double rel = 0.0, dmax = 0.0, rmax = 0.0;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    const double d = fabs(g[j] - r[j]), m = fabs(r[j]);
    rel = fmax(rel, m > 0.0 ? d / m : (d > 0.0 ? INFINITY : 0.0));
    dmax = fmax(dmax, d);
    rmax = fmax(rmax, m);
  }
  rel = block_reduce<true>(rel, sh);
  dmax = block_reduce<true>(dmax, sh);
  rmax = block_reduce<true>(rmax, sh);
  if (threadIdx.x == 0) {
    out[3 * a] = rel;
    out[3 * a + 1] = rmax > 0.0 ? dmax / rmax : dmax;
    out[3 * a + 2] = rmax;
  }
}

// compare.py:50-67 for one angle per block: d0 = computed curve, d1 = reference
// curve, n0 = ||d0||_2 (1 when 0), e0 = ||d0 - d1||_2; out[2a] = e0, out[2a+1] = n0.
// The script's printed values are e0 / max_a n0 and e0 / n0 (formed on the host).
__global__ void __launch_bounds__(256) k_curve_distance(const double* __restrict__ comp,
                                                        const double* __restrict__ ref, int nb,
                                                        double* __restrict__ out) {
  __shared__ double sh[32];
  const int a = blockIdx.x;
  const double* c = comp + (size_t)a * nb;
  const double* r = ref + (size_t)a * nb;
  double e = 0.0, n = 0.0;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
    const double d = c[j] - r[j];
    e = fma(d, d, e);
    n = fma(c[j], c[j], n);
  }
  e = block_reduce<false>(e, sh);
  n = block_reduce<false>(n, sh);
  if (threadIdx.x == 0) {
    const double n0 = sqrt(n);
    out[2 * a] = sqrt(e);
    out[2 * a + 1] = n0 == 0.0 ? 1.0 : n0;
  }
}

// domainsum.f90:58-106: s2[a][ibr] = sum over domains d (in order) and over the
// beams ib of d that rotate onto beam ibr of the reference domain (in order) of
// f2_d[a][ib] * w_d, each product rounded before the addition as the reference
// forms it.  One thread per (angle, reference beam).
__global__ void k_domain_sum(const DomainSumArgs args, int nang, int mb, double* __restrict__ s2) {
  const int ibr = blockIdx.x * blockDim.x + threadIdx.x, a = blockIdx.y;
  if (ibr >= mb || a >= nang) return;
  double s = 0.0;
  for (int d = 0; d < args.ndom; ++d) {
    const double* f = args.f2[d] + (size_t)a * args.nb[d];
    const int b0 = args.start[d * (mb + 1) + ibr], b1 = args.start[d * (mb + 1) + ibr + 1];
    for (int q = b0; q < b1; ++q) s = __dadd_rn(s, __dmul_rn(f[args.list[q]], args.w[d]));
  }
  s2[(size_t)a * mb + ibr] = s;
}

}  // namespace

void launch_domain_sum(const DomainSumArgs& args, int nang, int mb, double* s2, cudaStream_t st) {
  if (nang > 0 && mb > 0) k_domain_sum<<<dim3((mb + 127) / 128, nang), 128, 0, st>>>(args, nang, mb, s2);
}

void launch_curve_errors(const double* got, const double* ref, int nang, int nb, double* out,
                         cudaStream_t st) {
  if (nang > 0) k_curve_errors<<<nang, 256, 0, st>>>(got, ref, nb, out);
}

void launch_curve_distance(const double* comp, const double* ref, int nang, int nb, double* out,
                           cudaStream_t st) {
  if (nang > 0) k_curve_distance<<<nang, 256, 0, st>>>(comp, ref, nb, out);
}

}  // namespace trhepd
