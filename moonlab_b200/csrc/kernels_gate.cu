// kernels_gate.cu -- one full-state HBM sweep per gate (the engine's eager
// path, used for a single gate or when a tile pass cannot hold the gate).
//
// Work is enumerated only over the amplitudes a gate touches: a gate with c
// controls visits 2^(n-c) amplitudes (pairs / quads / diagonal entries), so
// a controlled gate moves 2*16*2^(n-c) bytes (complex128), not 2*16*2^n.
// Each thread issues ITEMS independent 16-byte loads before any store so
// that enough bytes are in flight to cover HBM latency.
#include <algorithm>
#include <cstdio>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 4;

struct GateParams {
  int32_t kind;      // MLB_OP_* after host canonicalisation
  int32_t t, t2;
  int32_t np;        // number of inserted zero positions
  uint64_t cmask;    // bits forced to 1 (controls; PHASE mask)
  uint64_t items;    // 2^(n - np)
  uint8_t pos[64];   // ascending insert positions
  double m[32];
  int32_t real_matrix;
};

template <typename Real>
__global__ void __launch_bounds__(kThreads) k_pair(typename Cplx<Real>::T* __restrict__ amp,
                                                   const GateParams p) {
  using A = typename Cplx<Real>::T;
  const uint64_t stride = (uint64_t)gridDim.x * kThreads * kItems;
  const uint64_t tb = 1ull << p.t;
  const A m00 = ld_m<Real>(p.m, 0), m01 = ld_m<Real>(p.m, 1);
  const A m10 = ld_m<Real>(p.m, 2), m11 = ld_m<Real>(p.m, 3);
  for (uint64_t base = (uint64_t)blockIdx.x * kThreads * kItems + threadIdx.x; base < p.items;
       base += stride) {
    uint64_t i0[kItems];
    A a0[kItems], a1[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      const uint64_t j = base + (uint64_t)k * kThreads;
      i0[k] = j < p.items ? (insert_zeros(j, p.pos, p.np) | p.cmask) : ~0ull;
      if (i0[k] != ~0ull) { a0[k] = amp[i0[k]]; a1[k] = amp[i0[k] | tb]; }
    }
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      if (i0[k] == ~0ull) continue;
      A b0, b1;
      if (p.kind == MLB_OP_X) {
        b0 = a1[k]; b1 = a0[k];
      } else if (p.real_matrix) {
        b0 = {m00.x * a0[k].x + m01.x * a1[k].x, m00.x * a0[k].y + m01.x * a1[k].y};
        b1 = {m10.x * a0[k].x + m11.x * a1[k].x, m10.x * a0[k].y + m11.x * a1[k].y};
      } else {
        b0 = cmul2(m00, a0[k], m01, a1[k]);
        b1 = cmul2(m10, a0[k], m11, a1[k]);
      }
      amp[i0[k]] = b0;
      amp[i0[k] | tb] = b1;
    }
  }
}

template <typename Real>
__global__ void __launch_bounds__(kThreads) k_quad(typename Cplx<Real>::T* __restrict__ amp,
                                                   const GateParams p) {
  using A = typename Cplx<Real>::T;
  const uint64_t stride = (uint64_t)gridDim.x * kThreads;
  const uint64_t b0 = 1ull << p.t, b1 = 1ull << p.t2;
  for (uint64_t j = (uint64_t)blockIdx.x * kThreads + threadIdx.x; j < p.items; j += stride) {
    const uint64_t i = insert_zeros(j, p.pos, p.np) | p.cmask;
    if (p.kind == MLB_OP_SWAP) {
      const A x = amp[i | b0], y = amp[i | b1];
      amp[i | b0] = y;
      amp[i | b1] = x;
      continue;
    }
    A v[4] = {amp[i], amp[i | b0], amp[i | b1], amp[i | b0 | b1]};
    A w[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      A acc = {0, 0};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const A mm = ld_m<Real>(p.m, r * 4 + c);
        acc.x += mm.x * v[c].x - mm.y * v[c].y;
        acc.y += mm.x * v[c].y + mm.y * v[c].x;
      }
      w[r] = acc;
    }
    amp[i] = w[0];
    amp[i | b0] = w[1];
    amp[i | b1] = w[2];
    amp[i | b0 | b1] = w[3];
  }
}

// Diagonal gates: PHASE (multiply the masked subspace), DIAG1 (key on bit t,
// over the control subspace), ZZ (key on parity of bits t, t2; all amps).
template <typename Real>
__global__ void __launch_bounds__(kThreads) k_diag(typename Cplx<Real>::T* __restrict__ amp,
                                                   const GateParams p) {
  using A = typename Cplx<Real>::T;
  const uint64_t stride = (uint64_t)gridDim.x * kThreads * kItems;
  const A d0 = ld_m<Real>(p.m, 0), d1 = ld_m<Real>(p.m, 1);
  const uint64_t zzmask = (1ull << p.t) | (p.t2 >= 0 ? (1ull << p.t2) : 0ull);
  for (uint64_t base = (uint64_t)blockIdx.x * kThreads * kItems + threadIdx.x; base < p.items;
       base += stride) {
    uint64_t idx[kItems];
    A a[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      const uint64_t j = base + (uint64_t)k * kThreads;
      idx[k] = j < p.items ? (insert_zeros(j, p.pos, p.np) | p.cmask) : ~0ull;
      if (idx[k] != ~0ull) a[k] = amp[idx[k]];
    }
#pragma unroll
    for (int k = 0; k < kItems; k++) {
      if (idx[k] == ~0ull) continue;
      A f;
      if (p.kind == MLB_OP_PHASE) f = d0;
      else if (p.kind == MLB_OP_DIAG1) f = ((idx[k] >> p.t) & 1ull) ? d1 : d0;
      else f = parity64(idx[k] & zzmask) ? d1 : d0;  // ZZ
      amp[idx[k]] = cmul(f, a[k]);
    }
  }
}

template <typename Real>
__global__ void k_init_zero(typename Cplx<Real>::T* __restrict__ amp, uint64_t dim) {
  using A = typename Cplx<Real>::T;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride)
    amp[i] = (i == 0) ? A{1, 0} : A{0, 0};
}

template <typename D, typename S>
__global__ void k_convert(D* __restrict__ dst, const S* __restrict__ src, uint64_t dim) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
    const S v = src[i];
    dst[i] = {(decltype(dst[i].x))v.x, (decltype(dst[i].y))v.y};
  }
}

int grid_for(uint64_t items, int per_block) {
  uint64_t b = (items + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > 148ull * 32) b = 148ull * 32;
  return (int)b;
}

void sort_unique(uint8_t* pos, int& np) {
  std::sort(pos, pos + np);
  np = (int)(std::unique(pos, pos + np) - pos);
}

}  // namespace

// Launch one eager gate.  Canonicalisation (host): DIAG1 whose |0> entry is 1
// becomes PHASE on the target=1 subspace; a 2Q gate whose matrix is the SWAP
// permutation becomes SWAP.
int launch_gate(int dtype, void* amp, int n, const mlb_op_t& op, cudaStream_t stream) {
  GateParams p{};
  p.kind = op.kind;
  p.t = op.target;
  p.t2 = op.target2;
  p.cmask = op.cmask;
  for (int k = 0; k < 32; k++) p.m[k] = op.m[k];
  int np = 0;
  for (int b = 0; b < n; b++)
    if (op.cmask >> b & 1ull) p.pos[np++] = (uint8_t)b;
  bool pair = false, quad = false;
  switch (op.kind) {
    case MLB_OP_1Q:
    case MLB_OP_X:
      p.pos[np++] = (uint8_t)op.target;
      pair = true;
      p.real_matrix = 1;
      for (int k = 1; k < 8; k += 2)
        if (op.m[k] != 0.0) p.real_matrix = 0;
      break;
    case MLB_OP_2Q:
    case MLB_OP_SWAP:
      p.pos[np++] = (uint8_t)op.target;
      p.pos[np++] = (uint8_t)op.target2;
      quad = true;
      break;
    case MLB_OP_DIAG1:
      if (op.m[0] == 1.0 && op.m[1] == 0.0) {  // phase on the target=1 half only
        p.kind = MLB_OP_PHASE;
        p.cmask |= 1ull << op.target;
        p.pos[np++] = (uint8_t)op.target;
        p.m[0] = op.m[2];
        p.m[1] = op.m[3];
      }
      break;
    case MLB_OP_PHASE:
      break;  // mask bits already in pos via cmask
    case MLB_OP_ZZ:
      p.m[2] = op.m[2];
      p.m[3] = op.m[3];
      break;
    default:
      return MLB_ERR_INVALID_ARG;
  }
  sort_unique(p.pos, np);
  p.np = np;
  p.items = 1ull << (n - np);
  const int per_block = kThreads * ((pair || !quad) ? kItems : 1);
  const int grid = grid_for(p.items, per_block);
  if (dtype == MLB_C128) {
    auto* a = reinterpret_cast<double2*>(amp);
    if (pair) k_pair<double><<<grid, kThreads, 0, stream>>>(a, p);
    else if (quad) k_quad<double><<<grid, kThreads, 0, stream>>>(a, p);
    else k_diag<double><<<grid, kThreads, 0, stream>>>(a, p);
  } else {
    auto* a = reinterpret_cast<float2*>(amp);
    if (pair) k_pair<float><<<grid, kThreads, 0, stream>>>(a, p);
    else if (quad) k_quad<float><<<grid, kThreads, 0, stream>>>(a, p);
    else k_diag<float><<<grid, kThreads, 0, stream>>>(a, p);
  }
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

int launch_init_zero(int dtype, void* amp, int n, cudaStream_t stream) {
  const uint64_t dim = 1ull << n;
  const int grid = grid_for(dim, 256);
  if (dtype == MLB_C128) k_init_zero<double><<<grid, 256, 0, stream>>>((double2*)amp, dim);
  else k_init_zero<float><<<grid, 256, 0, stream>>>((float2*)amp, dim);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

int launch_convert(int dst_dtype, void* dst, int src_dtype, const void* src, uint64_t dim,
                   cudaStream_t stream) {
  const int grid = grid_for(dim, 256);
  if (dst_dtype == MLB_C64 && src_dtype == MLB_C128)
    k_convert<float2, double2><<<grid, 256, 0, stream>>>((float2*)dst, (const double2*)src, dim);
  else if (dst_dtype == MLB_C128 && src_dtype == MLB_C64)
    k_convert<double2, float2><<<grid, 256, 0, stream>>>((double2*)dst, (const float2*)src, dim);
  else
    return MLB_ERR_INVALID_ARG;
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb
