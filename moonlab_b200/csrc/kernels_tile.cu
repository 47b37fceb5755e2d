// kernels_tile.cu -- multi-gate tile passes.
//
// One pass reads the whole state once and writes it once, applying a run of
// gates in between.  A tile is 2^(L+H) amplitudes: L contiguous low qubits
// (L=5: 512-byte runs for complex128, 256 bytes for complex64, so global
// loads and stores are fully coalesced 16/8-byte accesses) times the 2^H
// combinations of H chosen high qubits.  Tiles are enumerated over the
// remaining n-L-H qubits by a persistent grid sized to the SM count.
//
// Inside a tile the ops are grouped into segments: consecutive ops whose
// non-diagonal targets span at most R local bits.  For a segment each
// thread gathers a 2^R-amplitude group into registers, applies every op of
// the segment there, and scatters it back: one shared-memory round trip per
// segment instead of one per gate.  Controls and diagonal phases are
// evaluated per amplitude from its tile-local index; controls or diagonal
// qubits that lie outside the tile are constant over the tile and are
// evaluated once on the tile's base index.  Shared memory is XOR-swizzled on
// 128-byte rows so that group gathers of any stride are bank-conflict free.
#include <cstdio>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

template <typename Real> struct TileCfg;
template <> struct TileCfg<double> {  // complex128: 2^12 amps = 64 KiB per CTA
  static constexpr int TB = 12, RB = 3, NT = 256, MINB = 2, SW_SHIFT = 3, SW_MASK = 7;
};
template <> struct TileCfg<float> {   // complex64: 2^13 amps = 64 KiB per CTA
  static constexpr int TB = 13, RB = 4, NT = 256, MINB = 2, SW_SHIFT = 4, SW_MASK = 15;
};

// Tile-local index of register slot k of the current group: the group base
// with register bit b set for every set bit b of k.  k is a compile-time
// constant inside the unrolled loops, so this folds to a few ORs.
template <int RB>
struct Loc {
  uint32_t gb;
  uint32_t bm[RB];
  __device__ __forceinline__ uint32_t operator()(int k) const {
    uint32_t r = gb;
#pragma unroll
    for (int b = 0; b < RB; b++)
      if (k >> b & 1) r |= bm[b];
    return r;
  }
};

template <typename Real>
__device__ __forceinline__ uint32_t swz(uint32_t e) {
  return e ^ ((e >> TileCfg<Real>::SW_SHIFT) & TileCfg<Real>::SW_MASK);
}

// Apply one non-dense op to the register group.  RT / RT2 are compile-time
// register-bit positions so the amplitude array stays in registers.
template <typename Real, int G, int RT, int RBITS = (G == 16 ? 4 : G == 8 ? 3 : G == 4 ? 2 : G == 2 ? 1 : 5)>
__device__ __forceinline__ void pair_op(typename Cplx<Real>::T (&v)[G], const Loc<RBITS>& loc,
                                        const DevOp& op) {
  using A = typename Cplx<Real>::T;
  const A m00 = ld_m<Real>(op.m, 0), m01 = ld_m<Real>(op.m, 1);
  const A m10 = ld_m<Real>(op.m, 2), m11 = ld_m<Real>(op.m, 3);
#pragma unroll
  for (int k = 0; k < G; k++) {
    if (k & (1 << RT)) continue;
    const int k1 = k | (1 << RT);
    if ((loc(k) & op.lcmask) != op.lcmask) continue;
    const A a0 = v[k], a1 = v[k1];
    if (op.kind == DOP_X) {
      v[k] = a1;
      v[k1] = a0;
    } else if (op.kind == DOP_1Q_REAL) {
      v[k] = {m00.x * a0.x + m01.x * a1.x, m00.x * a0.y + m01.x * a1.y};
      v[k1] = {m10.x * a0.x + m11.x * a1.x, m10.x * a0.y + m11.x * a1.y};
    } else {
      v[k] = cmul2(m00, a0, m01, a1);
      v[k1] = cmul2(m10, a0, m11, a1);
    }
  }
}

template <typename Real, int G, int RT, int RT2, int RBITS = (G == 16 ? 4 : G == 8 ? 3 : G == 4 ? 2 : G == 2 ? 1 : 5)>
__device__ __forceinline__ void quad_op(typename Cplx<Real>::T (&v)[G], const Loc<RBITS>& loc,
                                        const DevOp& op) {
  using A = typename Cplx<Real>::T;
  constexpr int B0 = 1 << RT, B1 = 1 << RT2;
#pragma unroll
  for (int k = 0; k < G; k++) {
    if (k & (B0 | B1)) continue;
    if ((loc(k) & op.lcmask) != op.lcmask) continue;
    if (op.kind == DOP_SWAP) {
      const A t = v[k | B0];
      v[k | B0] = v[k | B1];
      v[k | B1] = t;
      continue;
    }
    const A x[4] = {v[k], v[k | B0], v[k | B1], v[k | B0 | B1]};
    A y[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      A acc = {0, 0};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const A mm = ld_m<Real>(op.m, r * 4 + c);
        acc.x += mm.x * x[c].x - mm.y * x[c].y;
        acc.y += mm.x * x[c].y + mm.y * x[c].x;
      }
      y[r] = acc;
    }
    v[k] = y[0];
    v[k | B0] = y[1];
    v[k | B1] = y[2];
    v[k | B0 | B1] = y[3];
  }
}

template <typename Real, int G, int RBITS = (G == 16 ? 4 : G == 8 ? 3 : G == 4 ? 2 : G == 2 ? 1 : 5)>
__device__ __forceinline__ void diag_op(typename Cplx<Real>::T (&v)[G], const Loc<RBITS>& loc,
                                        const DevOp& op, uint64_t tile_base) {
  using A = typename Cplx<Real>::T;
  const A d0 = ld_m<Real>(op.m, 0), d1 = ld_m<Real>(op.m, 1);
  if (op.kind == DOP_PHASE) {
    if ((tile_base & op.omask) != op.omask) return;
#pragma unroll
    for (int k = 0; k < G; k++)
      if ((loc(k) & op.lmask) == op.lmask) v[k] = cmul(d0, v[k]);
  } else if (op.kind == DOP_DIAG1) {
    const int out_bit = (tile_base & op.omask) ? 1 : 0;
#pragma unroll
    for (int k = 0; k < G; k++) {
      if ((loc(k) & op.lcmask) != op.lcmask) continue;
      const int b = op.lt >= 0 ? (int)((loc(k) >> op.lt) & 1u) : out_bit;
      v[k] = cmul(b ? d1 : d0, v[k]);
    }
  } else {  // DOP_ZZ
    const int po = parity64(tile_base & op.omask);
#pragma unroll
    for (int k = 0; k < G; k++) {
      const int par = (__popc(loc(k) & op.lmask) & 1) ^ po;
      v[k] = cmul(par ? d1 : d0, v[k]);
    }
  }
}

// Dense 2^nb x 2^nb block on the whole register group (complex64 fused path,
// CUDA-core version).  Matrix rows/cols follow the register-bit order.
template <typename Real, int G>
__device__ __forceinline__ void dense_op(typename Cplx<Real>::T (&v)[G], int nb,
                                         const DevOp& op, const float2* __restrict__ mats) {
  using A = typename Cplx<Real>::T;
  const int d = 1 << nb;
  const float2* M = mats + op.mat_off;
  A y[G];
#pragma unroll
  for (int r = 0; r < G; r++) {
    A acc = {0, 0};
    if (r < d) {
#pragma unroll
      for (int c = 0; c < G; c++) {
        if (c < d) {
          const float2 mm = __ldg(&M[r * d + c]);
          acc.x += (Real)mm.x * v[c].x - (Real)mm.y * v[c].y;
          acc.y += (Real)mm.x * v[c].y + (Real)mm.y * v[c].x;
        }
      }
    }
    y[r] = acc;
  }
#pragma unroll
  for (int r = 0; r < G; r++)
    if (r < d) v[r] = y[r];
}

template <typename Real, int G, int RBITS = (G == 16 ? 4 : G == 8 ? 3 : G == 4 ? 2 : G == 2 ? 1 : 5)>
__device__ __forceinline__ void apply_op(typename Cplx<Real>::T (&v)[G], const Loc<RBITS>& loc,
                                      const DevOp& op, uint64_t tile_base, int nb,
                                      const float2* __restrict__ mats) {
  switch (op.kind) {
    case DOP_1Q_GEN:
    case DOP_1Q_REAL:
    case DOP_X:
      switch (op.rt) {
        case 0: pair_op<Real, G, 0>(v, loc, op); break;
        case 1: if constexpr (G > 2) pair_op<Real, G, 1>(v, loc, op); break;
        case 2: if constexpr (G > 4) pair_op<Real, G, 2>(v, loc, op); break;
        case 3: if constexpr (G > 8) pair_op<Real, G, 3>(v, loc, op); break;
        case 4: if constexpr (G > 16) pair_op<Real, G, 4>(v, loc, op); break;
      }
      break;
    case DOP_2Q_GEN:
    case DOP_SWAP: {
      const int code = op.rt * 8 + op.rt2;
#define MLB_Q(a, b) \
  case a * 8 + b:   \
    if constexpr (G > (1 << a) && G > (1 << b)) quad_op<Real, G, a, b>(v, loc, op); \
    break;
      switch (code) {
        MLB_Q(0, 1) MLB_Q(0, 2) MLB_Q(0, 3) MLB_Q(1, 0) MLB_Q(1, 2) MLB_Q(1, 3)
        MLB_Q(2, 0) MLB_Q(2, 1) MLB_Q(2, 3) MLB_Q(3, 0) MLB_Q(3, 1) MLB_Q(3, 2)
      }
#undef MLB_Q
      break;
    }
    case DOP_DIAG1:
    case DOP_PHASE:
    case DOP_ZZ:
      diag_op<Real, G>(v, loc, op, tile_base);
      break;
    case DOP_DENSE:
      dense_op<Real, G>(v, nb, op, mats);
      break;
  }
}

template <typename Real>
__global__ void __launch_bounds__(TileCfg<Real>::NT, TileCfg<Real>::MINB)
    k_tile(typename Cplx<Real>::T* __restrict__ amp, const DevPass pass,
           const DevSegment* __restrict__ segs, const DevOp* __restrict__ ops,
           const float2* __restrict__ mats) {
  using A = typename Cplx<Real>::T;
  constexpr int NT = TileCfg<Real>::NT, RB = TileCfg<Real>::RB, G = 1 << RB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* sm = reinterpret_cast<A*>(smem_raw);
  __shared__ uint64_t rowoff[1 << (TileCfg<Real>::TB - 5)];

  const int L = pass.L, H = pass.H;
  const uint32_t tile_amps = 1u << (L + H);
  const uint32_t lmask_low = (1u << L) - 1u;
  for (uint32_t r = threadIdx.x; r < (1u << H); r += NT) {
    uint64_t off = 0;
#pragma unroll
    for (int k = 0; k < kMaxHigh; k++)  // static indices: pass stays in parameter space
      if (k < H && (r >> k & 1u)) off |= 1ull << pass.high[k];
    rowoff[r] = off;
  }
  __syncthreads();

  for (uint64_t tile = blockIdx.x; tile < pass.num_tiles; tile += gridDim.x) {
    const uint64_t tile_base = pdep64(tile, pass.tile_free_mask);
    // HBM -> shared (coalesced rows of 2^L amplitudes)
#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < tile_amps; e += NT) {
      const uint64_t g = tile_base | rowoff[e >> L] | (e & lmask_low);
      sm[swz<Real>(e)] = amp[g];
    }
    __syncthreads();

    for (int s = 0; s < pass.num_segments; s++) {
      const DevSegment& seg = segs[s];
      const int nb = seg.nbits;
      Loc<RB> lc;
#pragma unroll
      for (int b = 0; b < RB; b++) lc.bm[b] = b < nb ? (1u << seg.bits[b]) : 0u;
      const uint32_t groups = tile_amps >> nb;
      for (uint32_t gi = threadIdx.x; gi < groups; gi += NT) {
        uint32_t gb = gi;
        for (int b = 0; b < nb; b++) {
          const uint32_t p = seg.bits[b];
          gb = ((gb >> p) << (p + 1)) | (gb & ((1u << p) - 1u));
        }
        lc.gb = gb;
        A v[G];
#pragma unroll
        for (int k = 0; k < G; k++)
          if (k < (1 << nb)) v[k] = sm[swz<Real>(lc(k))];
        for (int o = seg.op_begin; o < seg.op_end; o++) {
          const DevOp& op = ops[o];
          if ((tile_base & op.ocmask) != op.ocmask) continue;
          apply_op<Real, G>(v, lc, op, tile_base, nb, mats);
        }
#pragma unroll
        for (int k = 0; k < G; k++)
          if (k < (1 << nb)) sm[swz<Real>(lc(k))] = v[k];
      }
      __syncthreads();
    }

    // shared -> HBM
#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < tile_amps; e += NT) {
      const uint64_t g = tile_base | rowoff[e >> L] | (e & lmask_low);
      amp[g] = sm[swz<Real>(e)];
    }
    __syncthreads();
  }
}

template <typename Real>
int launch_tile_t(void* amp, const DevPass& pass, const DevSegment* d_segs, const DevOp* d_ops,
                  const float2* d_mats, int num_sms, cudaStream_t stream) {
  using A = typename Cplx<Real>::T;
  constexpr int NT = TileCfg<Real>::NT;
  const size_t smem = sizeof(A) << (pass.L + pass.H);
  static bool attr_set = false;
  const size_t max_smem = sizeof(A) << TileCfg<Real>::TB;
  if (!attr_set) {
    cudaFuncSetAttribute(k_tile<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    attr_set = true;
  }
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile<Real>, NT, smem);
  if (per_sm < 1) per_sm = 1;
  uint64_t grid = (uint64_t)num_sms * per_sm;
  if (grid > pass.num_tiles) grid = pass.num_tiles;
  k_tile<Real><<<(unsigned)grid, NT, smem, stream>>>(reinterpret_cast<A*>(amp), pass, d_segs,
                                                     d_ops, d_mats);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace

int launch_tile_pass(int dtype, void* amp, const DevPass& pass, const DevSegment* d_segs,
                     const DevOp* d_ops, const float2* d_mats, int num_sms, cudaStream_t stream) {
  if (dtype == MLB_C128)
    return launch_tile_t<double>(amp, pass, d_segs, d_ops, d_mats, num_sms, stream);
  return launch_tile_t<float>(amp, pass, d_segs, d_ops, d_mats, num_sms, stream);
}

}  // namespace mlb
