// Rocking-curve epilogues on the device (curves.cu).
#pragma once
#include <cuda_runtime.h>

namespace trhepd {

// Per curve a of got/ref (nang x nb): out[3a] max relative error over every spot,
// out[3a+1] max |got - ref| / max |ref|, out[3a+2] max |ref|.
void launch_curve_errors(const double* got, const double* ref, int nang, int nb, double* out,
                         cudaStream_t st);
// compare.py's per-angle distance: out[2a] = ||comp_a - ref_a||_2, out[2a+1] = ||comp_a||_2
// (1 when zero).
void launch_curve_distance(const double* comp, const double* ref, int nang, int nb, double* out,
                           cudaStream_t st);

// Weighted sum of rotated-domain rocking curves (domainsum.f90): per domain d its
// intensities f2[d] (nang x nb[d], device), weight w[d], and for every beam ibr of
// the reference domain the beams of d that rotate onto it: list[start[d*(mb+1) + ibr]
// .. start[d*(mb+1) + ibr + 1]) (device, increasing order).  At most kMaxDomains.
constexpr int kMaxDomains = 16;
struct DomainSumArgs {
  int ndom;
  const double* f2[kMaxDomains];
  int nb[kMaxDomains];
  double w[kMaxDomains];
  const int* start;  // ndom x (mb + 1) offsets into list
  const int* list;
};
void launch_domain_sum(const DomainSumArgs& args, int nang, int mb, double* s2, cudaStream_t st);

}  // namespace trhepd
