// kernels_common.cuh -- complex arithmetic and index helpers for the
// state-vector kernels.  Amplitudes are double2 (complex128) or float2
// (complex64); `Real` is the component type.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace mlb {

template <typename Real> struct Cplx;
template <> struct Cplx<double> { using T = double2; };
template <> struct Cplx<float>  { using T = float2; };

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2  mk(float x, float y)   { return make_float2(x, y); }

template <typename A> __device__ __forceinline__ A cmul(A a, A b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a*b + c*d (complex), the 2x2 row product.
template <typename A> __device__ __forceinline__ A cmul2(A a, A b, A c, A d) {
  return {a.x * b.x - a.y * b.y + c.x * d.x - c.y * d.y,
          a.x * b.y + a.y * b.x + c.x * d.y + c.y * d.x};
}

template <typename Real>
__device__ __forceinline__ typename Cplx<Real>::T ld_m(const double* m, int k) {
  return {(Real)m[2 * k], (Real)m[2 * k + 1]};
}

// Insert a zero bit at each of the ascending positions pos[0..np).
__device__ __forceinline__ uint64_t insert_zeros(uint64_t j, const uint8_t* pos, int np) {
#pragma unroll 4
  for (int k = 0; k < np; k++) {
    const uint64_t p = pos[k];
    const uint64_t lo = j & ((1ull << p) - 1ull);
    j = ((j >> p) << (p + 1)) | lo;
  }
  return j;
}

// Deposit the low bits of j into the set bits of mask (software pdep).
__device__ __forceinline__ uint64_t pdep64(uint64_t j, uint64_t mask) {
  uint64_t r = 0;
  while (mask) {
    const uint64_t low = mask & (~mask + 1ull);
    if (j & 1ull) r |= low;
    j >>= 1;
    mask ^= low;
  }
  return r;
}

__device__ __forceinline__ int parity64(uint64_t x) { return __popcll(x) & 1; }

}  // namespace mlb
