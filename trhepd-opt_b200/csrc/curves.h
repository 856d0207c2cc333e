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

}  // namespace trhepd
