// Shared device helpers for the multislice surface solve (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace trhepd {

struct cd {  // complex double, layout-compatible with Fortran complex(8) / double _Complex
  double x, y;
};

__host__ __device__ __forceinline__ cd mk(double x, double y) { return cd{x, y}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a) { return cd{-a.x, -a.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) {
  return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ cd conj(cd a) { return cd{a.x, -a.y}; }
// acc + a b and acc - a b as four fused multiply-adds (rounds differently from
// acc + (a * b) with the product formed first)
__host__ __device__ __forceinline__ cd cfma(cd a, cd b, cd acc) {
  return cd{fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y))};
}
__host__ __device__ __forceinline__ cd cfms(cd a, cd b, cd acc) {
  return cd{fma(-a.x, b.x, fma(a.y, b.y, acc.x)), fma(-a.x, b.y, fma(-a.y, b.x, acc.y))};
}
__host__ __device__ __forceinline__ double cabs1(cd a) { return fabs(a.x) + fabs(a.y); }
// a / b with the scaling of Smith's algorithm
__host__ __device__ __forceinline__ cd cdiv(cd a, cd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, den = b.x + b.y * r;
    return cd{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
  } else {
    double r = b.x / b.y, den = b.x * r + b.y;
    return cd{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
  }
}

__host__ __device__ __forceinline__ int ceil_div(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ __forceinline__ int round_up(int a, int b) { return ceil_div(a, b) * b; }

// Device status word bits (read back by the host after each solve).
enum : unsigned {
  kStatusNonFinite = 1u << 0,
  kStatusZeroPivot = 1u << 1,
  kStatusTimeout = 1u << 2,
};

}  // namespace trhepd
