// kernels_tile.cu -- multi-gate tile passes.
//
// One pass reads the whole state once and writes it once, applying a run of
// gates in between.  A tile is 2^(L+H) amplitudes: L contiguous low qubits
// (complex128: L = 2, 64-byte rows, 12-bit tiles of 64 KiB; complex64: L = 5,
// 256-byte rows, 13-bit tiles of 64 KiB; global loads and stores are whole
// 16/8-byte accesses in full rows) times the 2^H combinations of H chosen
// high qubits.  Tiles are enumerated over the remaining n-L-H qubits by a
// persistent grid sized to the SM count.
//
// Inside a tile the ops are grouped into segments: consecutive ops whose
// non-diagonal targets span at most R local bits.  For a segment each
// thread gathers two 2^R-amplitude groups into registers, applies every op
// of the segment there (the two groups interleaved for instruction-level
// parallelism), and scatters them back: one shared-memory round trip per
// segment instead of one per gate.  The pass's ops are decoded once per CTA
// into a compact shared-memory program (matrices pre-converted to the state's
// precision), and the tile-constant part of every op -- controls, phase
// masks and diagonal keys on qubits outside the tile -- is evaluated once
// per tile.  Shared memory is XOR-swizzled on 128-byte rows so that group
// gathers of most strides are bank-conflict free (complex128: every tile bit
// moves the bank group; see tile_swz16).
//
// complex128 segments that the host multiplied into one 16x16 complex matrix
// (dense.h; mode 2) run on the FP64 tensor cores instead: the tile's 256
// groups of 16 amplitudes are the columns of a 16 x 256 complex block, each
// warp takes two column tiles of 8 groups at a time, loads them as the B
// fragments of 4 k-steps (four 16-byte loads per lane per column tile), runs
// 3 real products x 2 m-tiles x 4 k-steps = 24 mma.sync m8n8k4 f64 per column
// tile (Gauss's three-product complex multiplication) with the matrix
// fragments in registers and stores the results back in place (four 16-byte
// stores per lane per column tile).  Gate by gate, a
// segment's ~12 ops cost about as many FP64 multiply-adds as the dense
// product (48 per amplitude) but spend two thirds of their instruction issue
// on addressing, dispatch and register moves; one DMMA is 256 of them.
#include <atomic>
#include <cstdio>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

template <typename Real> struct TileCfg;
template <> struct TileCfg<double> {  // complex128: 2^12 amps = 64 KiB per CTA, two CTAs of 4 warps per SM
  static constexpr int TB = kTileBitsC128, RB = 4, NT = 128, MINB = 2, SW_SHIFT = 3, SW_MASK = 7, GPT = 1;
  static constexpr int LOW = kLowBitsC128;
};
template <> struct TileCfg<float> {   // complex64: 2^13 amps = 64 KiB per CTA
  static constexpr int TB = 13, RB = 4, NT = 256, MINB = 2, SW_SHIFT = 4, SW_MASK = 15, GPT = 1;
  static constexpr int LOW = 5;
};
// GPT: register groups per thread per segment, interleaved for ILP.  LOW:
// contiguous low qubits of a tile of a state larger than one tile (rows).
// complex128 CTAs on one SM run independent tile sequences, so one CTA's
// loads and stores overlap the others' tensor-core work: two per SM in
// general, three in dense-only passes (a CTA of 4 warps keeps the FP64
// tensor pipe busy only together with others: with two per SM, the pipe
// starves while one of them is in its memory phase).

template <typename Real>
__device__ __forceinline__ uint32_t swz(uint32_t e) {
  if constexpr (sizeof(Real) == 8) return tile_swz16(e);  // shared with the dense segments' host tables
  return e ^ ((e >> TileCfg<Real>::SW_SHIFT) & TileCfg<Real>::SW_MASK);
}

// Compact op, decoded into shared memory at kernel start.
struct SmOp {
  uint8_t kind, rt, rt2, la;  // register bits (pair/quad), local key bit (31: none)
  uint8_t lb, ctrl, code, pad1;
  uint32_t lcmask;             // local control mask
  uint32_t lmask;              // local mask (PHASE)
  uint32_t mat;                // op index (matrix slot) or 2Q: global op index
};

// Tile-local index of register slot k of group base gb.
template <int RB>
struct Dep {
  uint32_t bm[RB];
  __device__ __forceinline__ uint32_t operator()(uint32_t gb, int k) const {
    uint32_t r = gb;
#pragma unroll
    for (int b = 0; b < RB; b++)
      if (k >> b & 1) r |= bm[b];
    return r;
  }
};

template <typename A, int G, int RB, int RT, int KIND, bool CTRL, int kGPT>
__device__ __forceinline__ void op_pair(A (&v)[kGPT][G], const uint32_t (&gb)[kGPT], const Dep<RB>& dep,
                                        const SmOp& op, const A* __restrict__ M) {
  A m00, m01, m10, m11;
  if (KIND != DOP_X) { m00 = M[0]; m01 = M[1]; m10 = M[2]; m11 = M[3]; }
#pragma unroll
  for (int g = 0; g < kGPT; g++) {
#pragma unroll
    for (int k = 0; k < G; k++) {
      if (k & (1 << RT)) continue;
      const int k1 = k | (1 << RT);
      if (CTRL && (dep(gb[g], k) & op.lcmask) != op.lcmask) continue;
      const A a0 = v[g][k], a1 = v[g][k1];
      if (KIND == DOP_X) {
        v[g][k] = a1;
        v[g][k1] = a0;
      } else if (KIND == DOP_1Q_REAL) {
        v[g][k] = {m00.x * a0.x + m01.x * a1.x, m00.x * a0.y + m01.x * a1.y};
        v[g][k1] = {m10.x * a0.x + m11.x * a1.x, m10.x * a0.y + m11.x * a1.y};
      } else {
        v[g][k] = cmul2(m00, a0, m01, a1);
        v[g][k1] = cmul2(m10, a0, m11, a1);
      }
    }
  }
}

template <typename A, int G, int RB, int RT, int RT2, bool CTRL, int kGPT>
__device__ __forceinline__ void op_swap(A (&v)[kGPT][G], const uint32_t (&gb)[kGPT], const Dep<RB>& dep,
                                        const SmOp& op) {
  constexpr int B0 = 1 << RT, B1 = 1 << RT2;
#pragma unroll
  for (int g = 0; g < kGPT; g++) {
#pragma unroll
    for (int k = 0; k < G; k++) {
      if (k & (B0 | B1)) continue;
      if (CTRL && (dep(gb[g], k) & op.lcmask) != op.lcmask) continue;
      const A t = v[g][k | B0];  // SWAP
      v[g][k | B0] = v[g][k | B1];
      v[g][k | B1] = t;
    }
  }
}

// A generic 4x4 op on local bits (l0 = low index bit, l1), applied directly
// in shared memory, one quad per thread iteration.
template <typename Real>
__device__ __forceinline__ void smem_quad(typename Cplx<Real>::T* sm, uint32_t tile_amps,
                                          const DevOp& d, int NT) {
  using A = typename Cplx<Real>::T;
  const uint32_t l0 = (uint32_t)d.lt, l1 = (uint32_t)d.k;
  const uint32_t lo = l0 < l1 ? l0 : l1, hi = l0 < l1 ? l1 : l0;
  const uint32_t b0 = 1u << l0, b1 = 1u << l1;
  const double* __restrict__ M = d.m;
  for (uint32_t q = threadIdx.x; q < (tile_amps >> 2); q += NT) {
    // matrix entries are re-read (L1) per quad: holding all 16 in registers
    // next to the kernel's amplitude groups would exceed the register budget
    asm volatile("" ::: "memory");
    uint32_t i = q;
    i = ((i >> lo) << (lo + 1)) | (i & ((1u << lo) - 1u));
    i = ((i >> hi) << (hi + 1)) | (i & ((1u << hi) - 1u));
    if ((i & d.lcmask) != d.lcmask) continue;
    const uint32_t idx[4] = {i, i | b0, i | b1, i | b0 | b1};
    A x[4], y[4];
#pragma unroll
    for (int c = 0; c < 4; c++) x[c] = sm[swz<Real>(idx[c])];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      A acc = {0, 0};
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const Real mr = (Real)M[(r * 4 + c) * 2], mi = (Real)M[(r * 4 + c) * 2 + 1];
        acc.x += mr * x[c].x - mi * x[c].y;
        acc.y += mr * x[c].y + mi * x[c].x;
      }
      y[r] = acc;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) sm[swz<Real>(idx[c])] = y[c];
  }
}

// DIAG1 / ZZ: f = M[key], key = bit la (xor bit lb) of the local index xor
// the tile-constant key.  PHASE: multiply by M[0] where the local mask holds.
template <typename A, int G, int RB, bool PHASE, bool CTRL, int kGPT>
__device__ __forceinline__ void op_diag(A (&v)[kGPT][G], const uint32_t (&gb)[kGPT], const Dep<RB>& dep,
                                        const SmOp& op, const A* __restrict__ M, uint32_t tkey) {
  const A d0 = M[0], d1 = M[1];
#pragma unroll
  for (int g = 0; g < kGPT; g++) {
#pragma unroll
    for (int k = 0; k < G; k++) {
      const uint32_t loc = dep(gb[g], k);
      if (PHASE) {
        if ((loc & op.lmask) == op.lmask) v[g][k] = cmul(d0, v[g][k]);
      } else {
        if (CTRL && (loc & op.lcmask) != op.lcmask) continue;
        const uint32_t key = ((loc >> op.la) ^ (loc >> op.lb) ^ tkey) & 1u;
        v[g][k] = cmul(key ? d1 : d0, v[g][k]);
      }
    }
  }
}

// Dispatch code of an op: one switch selects a fully specialised routine.
//   pair ops:  (kind 0..2) * 16 + rt * 2 + ctrl          -> 0 .. 47
//   swap:      64 + (rt * 4 + rt2) * 2 + ctrl            -> 64 .. 95
//   diag:      96 + phase * 2 + ctrl                     -> 96 .. 99
__host__ __device__ constexpr int code_pair(int kind, int rt, int ctrl) { return kind * 16 + rt * 2 + ctrl; }
__host__ __device__ constexpr int code_swap(int rt, int rt2, int ctrl) { return 64 + (rt * 4 + rt2) * 2 + ctrl; }
__host__ __device__ constexpr int code_diag(int phase, int ctrl) { return 96 + phase * 2 + ctrl; }

static_assert(kDenseMaxCondLoc <= 5, "dense segments: a column-tile pair (j, j + 1) must share its variant");

__device__ __forceinline__ void dmma_f64(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Mode-2 segment: every group of the tile times the segment's dense matrix
// U = R + iJ (the variant of this group's and tile's conditioning bits), as
// three real 16 x 16 products (Gauss): t1 = R xr, t2 = J xi,
// t3 = (R + J)(xr + xi); yr = t1 - t2, yi = t3 - t1 - t2.  Fragment layout
// of mma.sync m8n8k4 f64 (lane l, r = l >> 2, c = l & 3): A[r][c], B[c][r],
// D[r][2 c], D[r][2 c + 1]; the host stores R and J so that lane l's B
// operands are whole input slots 4 s + c of group r (re for t1, im for t2,
// their sum for t3) and its D results whole output slots r and 8 + r of
// groups 2 c and 2 c + 1.
template <int NT>
__device__ __forceinline__ void dense_segment(double2* __restrict__ sm, const DenseSegDev* __restrict__ sg,
                                              const double* __restrict__ frags, uint64_t tile_base) {
  constexpr int kWarps = NT / 32, kPerWarp = (1 << kDenseColBits) / kWarps;  // column tiles of 8 groups
  // warp w takes column tiles kPerWarp w .. + kPerWarp - 1: their conditioning
  // values (the top group-index bits) rarely change within a warp
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g8 = lane >> 2, q = lane & 3;
  const int nloc = sg->nloc, nout = sg->nout;
  uint32_t vout = 0;
  for (int j = 0; j < nout; j++) vout |= (uint32_t)((tile_base >> sg->obit[j]) & 1ull) << j;
  uint32_t boff[4];
#pragma unroll
  for (int t4 = 0; t4 < 4; t4++) boff[t4] = sg->amp_off[4 * t4 + q];
  const uint32_t doff0 = sg->amp_off[g8], doff1 = sg->amp_off[8 + g8];
  const uint32_t glb = sg->g_lo[g8], gld0 = sg->g_lo[2 * q], gld1 = sg->g_lo[2 * q + 1];
  const double* fseg = frags + sg->frag_off + lane;
  int cur = -1;
  double ar[8], aj[8], arj[8];  // fragment (i, s) at index 4 i + s; arj = ar + aj
  // two column tiles per step: 12 independent accumulator chains per warp
  // cover the DMMA latency; they differ only in bit 0 of j, so they share
  // their conditioning values (the top nloc <= 5 of j's 6 bits)
  // this warp's column-tile offsets, one per lane, passed along by shuffles
  // (no table read in the step's dependency chain)
  const uint32_t my_ghi = sg->g_hi[kPerWarp * warp + (lane % kPerWarp)];
#pragma unroll 1
  for (int u = 0; u < kPerWarp; u += 2) {
    const int j = kPerWarp * warp + u;  // column tiles j, j + 1: groups 8 j .. 8 j + 15
    const uint32_t ghi0 = __shfl_sync(0xffffffffu, my_ghi, u), ghi1 = __shfl_sync(0xffffffffu, my_ghi, u + 1);
    const int var = (nloc ? (j >> (kDenseColBits - nloc)) : 0) | (int)(vout << nloc);
    if (var != cur) {  // warp-uniform
      const double* f = fseg + (size_t)var * kDenseVarDoubles;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        ar[k] = __ldg(f + 32 * k);
        aj[k] = __ldg(f + 32 * (8 + k));
      }
#pragma unroll
      for (int k = 0; k < 8; k++) arj[k] = ar[k] + aj[k];  // R + J, once per variant
      cur = var;
    }
    double2 x0[4], x1[4];  // this step's B operands (two column tiles)
#pragma unroll
    for (int t4 = 0; t4 < 4; t4++) {
      x0[t4] = sm[ghi0 ^ glb ^ boff[t4]];
      x1[t4] = sm[ghi1 ^ glb ^ boff[t4]];
    }
    // [column tile][product][m-tile][column]
    double t[2][3][2][2];
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int p = 0; p < 3; p++)
#pragma unroll
        for (int i = 0; i < 2; i++) t[c][p][i][0] = t[c][p][i][1] = 0.0;
#pragma unroll
    for (int sk = 0; sk < 4; sk++) {
      const double s0 = x0[sk].x + x0[sk].y, s1 = x1[sk].x + x1[sk].y;
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int f = 4 * i + sk;
        dmma_f64(t[0][0][i][0], t[0][0][i][1], ar[f], x0[sk].x);
        dmma_f64(t[1][0][i][0], t[1][0][i][1], ar[f], x1[sk].x);
        dmma_f64(t[0][1][i][0], t[0][1][i][1], aj[f], x0[sk].y);
        dmma_f64(t[1][1][i][0], t[1][1][i][1], aj[f], x1[sk].y);
        const double af = arj[f];
        dmma_f64(t[0][2][i][0], t[0][2][i][1], af, s0);
        dmma_f64(t[1][2][i][0], t[1][2][i][1], af, s1);
      }
    }
    // in place: this warp's 16 groups are read above and by no other warp
    auto out = [&](int c, int i, int col) {
      const double t1 = t[c][0][i][col], t2 = t[c][1][i][col];
      return make_double2(t1 - t2, t[c][2][i][col] - t1 - t2);
    };
    sm[ghi0 ^ gld0 ^ doff0] = out(0, 0, 0);
    sm[ghi0 ^ gld0 ^ doff1] = out(0, 1, 0);
    sm[ghi0 ^ gld1 ^ doff0] = out(0, 0, 1);
    sm[ghi0 ^ gld1 ^ doff1] = out(0, 1, 1);
    sm[ghi1 ^ gld0 ^ doff0] = out(1, 0, 0);
    sm[ghi1 ^ gld0 ^ doff1] = out(1, 1, 0);
    sm[ghi1 ^ gld1 ^ doff0] = out(1, 0, 1);
    sm[ghi1 ^ gld1 ^ doff1] = out(1, 1, 1);
  }
}

// DENSE (complex128 passes whose segments all run dense): only the dense
// segment code, no op program to decode (fewer registers and less shared
// memory than the kernel that also runs gate-by-gate segments).
template <typename Real, bool DENSE>
__global__ void __launch_bounds__(TileCfg<Real>::NT, DENSE ? 3 : TileCfg<Real>::MINB)
    k_tile(typename Cplx<Real>::T* __restrict__ amp, const DevPass pass,
           const DevSegment* __restrict__ segs, const DevOp* __restrict__ ops,
           const DenseSegDev* __restrict__ dsegs, const double* __restrict__ frags) {
  using A = typename Cplx<Real>::T;
  constexpr int NT = TileCfg<Real>::NT, RB = TileCfg<Real>::RB, G = 1 << RB, kGPT = TileCfg<Real>::GPT;
  constexpr int TB = TileCfg<Real>::TB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* sm = reinterpret_cast<A*>(smem_raw);
  // global offsets of the tile's rows (its high-qubit combinations); rows
  // are 2^LOW amplitudes long
  __shared__ uint64_t rowoff[1 << (TileCfg<Real>::TB - TileCfg<Real>::LOW)];
  constexpr int kProg = DENSE ? 1 : kMaxPassOps;  // the op program (gate-by-gate segments)
  __shared__ SmOp sops[kProg];
  __shared__ A smat[kProg][4];
  __shared__ uint8_t ton[kProg];
  __shared__ uint8_t tkey[kProg];
  __shared__ DevSegment ssegs[DENSE ? 1 : kMaxPassSegs];
  // dense-only passes: two staging slots for the segments' offset tables
  // (application q reads slot q & 1 while application q + 1's is staged)
  // and the segments' dense indices; small enough for three CTAs per SM
  __shared__ DenseSegDev sdseg[DENSE ? 2 : 1];
  __shared__ uint16_t didx[DENSE ? kMaxPassSegs : 1];
  static_assert(sizeof(DenseSegDev) == 128, "staged as 32 words");

  const int L = pass.L, H = pass.H;
  const uint32_t tile_amps = 1u << (L + H);
  const uint32_t lmask_low = (1u << L) - 1u;
  const int nseg = pass.num_segments;
  const int op0 = segs[0].op_begin, nops = segs[nseg - 1].op_end - op0;

  // ---- prologue: row offsets, compact program ----
  for (uint32_t r = threadIdx.x; r < (1u << H); r += NT) {
    uint64_t off = 0;
#pragma unroll
    for (int k = 0; k < kMaxHigh; k++)  // static indices: pass stays in parameter space
      if (k < H && (r >> k & 1u)) off |= 1ull << pass.high[k];
    rowoff[r] = off;
  }
  if constexpr (DENSE) {
    for (int s = threadIdx.x; s < nseg; s += NT) didx[s] = (uint16_t)segs[s].dense;
    if (threadIdx.x < 32)
      reinterpret_cast<uint32_t*>(sdseg)[threadIdx.x] =
          reinterpret_cast<const uint32_t*>(dsegs + segs[0].dense)[threadIdx.x];
  } else {
    for (int s = threadIdx.x; s < nseg; s += NT) {
      DevSegment sg = segs[s];
      sg.op_begin -= op0;
      sg.op_end -= op0;
      ssegs[s] = sg;
    }
  }
  for (int o = threadIdx.x; o < (DENSE ? 0 : nops); o += NT) {
    const DevOp& d = ops[op0 + o];
    SmOp so;
    so.kind = (uint8_t)d.kind;
    so.rt = (uint8_t)(d.rt < 0 ? 0 : d.rt);
    so.rt2 = (uint8_t)(d.rt2 < 0 ? 0 : d.rt2);
    so.la = 31;
    so.lb = 31;
    so.ctrl = d.lcmask != 0;
    so.lcmask = d.lcmask;
    so.lmask = d.lmask;
    so.mat = (uint32_t)(op0 + o);
    if (d.kind == DOP_1Q_GEN || d.kind == DOP_1Q_REAL || d.kind == DOP_X)
      so.code = (uint8_t)code_pair(d.kind, so.rt, so.ctrl);
    else if (d.kind == DOP_SWAP)
      so.code = (uint8_t)code_swap(so.rt, so.rt2, so.ctrl);
    else
      so.code = (uint8_t)code_diag(d.kind == DOP_PHASE ? 1 : 0, so.ctrl);
    if (d.kind == DOP_DIAG1) {
      so.la = d.lt >= 0 ? (uint8_t)d.lt : 31;
    } else if (d.kind == DOP_ZZ) {
      // up to two local bits of lmask; the rest is tile-constant parity
      uint32_t lm = d.lmask;
      if (lm) { so.la = (uint8_t)(__ffs(lm) - 1); lm &= lm - 1; }
      if (lm) { so.lb = (uint8_t)(__ffs(lm) - 1); }
    }
    sops[o] = so;
#pragma unroll
    for (int k = 0; k < 4; k++) smat[o][k] = A{(Real)d.m[2 * k], (Real)d.m[2 * k + 1]};
  }
  __syncthreads();

  // Full tiles: the store of a tile and the load of the CTA's next tile share
  // one loop: each thread stores an element from its shared-memory slot and
  // refills that slot with the next tile's element by a 16/8-byte cp.async
  // (its own slot, read before, so no barrier), so the load latency overlaps
  // the stores instead of following them.
  const bool full = tile_amps == (1u << TB);
  const uint32_t sm_base = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
  // Row offset of element e = threadIdx.x + j NT of a full tile: NT is a
  // multiple of the row length 2^L (or the tile has no high bits and every
  // row offset is 0), so e >> L = (threadIdx.x >> L) | (j NT >> L) on
  // disjoint bits and the offset is this thread's part OR a part that is
  // the same for every thread (a broadcast read instead of a per-lane one).
  // Used for complex128 (measured 1.6 % faster there, 1.4 % slower for
  // complex64's 5-bit rows).
  const uint64_t my_row = rowoff[threadIdx.x >> L];
  auto row_of = [&](uint32_t e, int j) -> uint64_t {
    if constexpr (sizeof(Real) == 8) return my_row | rowoff[(uint32_t)(j * NT) >> L];
    else return rowoff[e >> L];
  };
  bool prefetched = false;
  uint32_t dq = 0;  // dense-only passes: segment applications so far (staging slot parity)
  for (uint64_t tile = blockIdx.x; tile < pass.num_tiles; tile += gridDim.x) {
    const uint64_t tile_base = pdep64(tile, pass.tile_free_mask);
    // tile-constant op predicates and keys
    for (int o = threadIdx.x; o < (DENSE ? 0 : nops); o += NT) {
      const DevOp& d = ops[op0 + o];
      bool on = (tile_base & d.ocmask) == d.ocmask;
      uint32_t key = 0;
      if (d.kind == DOP_PHASE) on = on && ((tile_base & d.omask) == d.omask);
      else key = (uint32_t)(__popcll(tile_base & d.omask) & 1);
      ton[o] = on;
      tkey[o] = (uint8_t)key;
    }
    // HBM -> shared (coalesced rows of 2^L amplitudes).  A full tile has a
    // compile-time trip count, so all of a thread's loads are in flight at once.
    if (prefetched) {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    } else if (full) {
      constexpr int PER = (1 << TB) / NT;
      A tmp[PER];
#pragma unroll
      for (int j = 0; j < PER; j++) {
        const uint32_t e = threadIdx.x + j * NT;
        tmp[j] = __ldcs(&amp[tile_base | row_of(e, j) | (e & lmask_low)]);
      }
#pragma unroll
      for (int j = 0; j < PER; j++) sm[swz<Real>(threadIdx.x + j * NT)] = tmp[j];
    } else {
      for (uint32_t e = threadIdx.x; e < tile_amps; e += NT) {
        const uint64_t gidx = tile_base | rowoff[e >> L] | (e & lmask_low);
        sm[swz<Real>(e)] = amp[gidx];
      }
    }
    __syncthreads();

    for (int s = 0; s < nseg; s++) {
      if constexpr (DENSE) {
        // stage the next application's table (the next segment, or segment 0
        // of the next tile) into the other slot; the barrier publishes it
        const int sn = s + 1 < nseg ? s + 1 : 0;
        uint32_t w = 0;
        if (threadIdx.x < 32) w = reinterpret_cast<const uint32_t*>(dsegs + didx[sn])[threadIdx.x];
        dense_segment<NT>(reinterpret_cast<double2*>(sm), sdseg + (dq & 1u), frags, tile_base);
        if (threadIdx.x < 32) reinterpret_cast<uint32_t*>(sdseg + ((dq + 1u) & 1u))[threadIdx.x] = w;
        dq++;
        __syncthreads();
        continue;
      }
      const DevSegment& seg = ssegs[s];
      if constexpr (sizeof(Real) == 8) {
        if (seg.mode == 2) {
          dense_segment<NT>(reinterpret_cast<double2*>(sm), dsegs + seg.dense, frags, tile_base);
          __syncthreads();
          continue;
        }
      }
      if constexpr (!DENSE) {
      if (seg.mode == 1) {
        const int o = seg.op_begin;
        if (ton[o]) smem_quad<Real>(sm, tile_amps, ops[op0 + o], NT);
        __syncthreads();
        continue;
      }
      const int nb = seg.nbits;
      Dep<RB> dep;
#pragma unroll
      for (int b = 0; b < RB; b++) dep.bm[b] = b < nb ? (1u << seg.bits[b]) : 0u;
      const uint32_t groups = tile_amps >> nb;
      for (uint32_t g0 = threadIdx.x; g0 < groups; g0 += NT * kGPT) {
        uint32_t gb[kGPT];
        bool valid[kGPT];
        A v[kGPT][G];
#pragma unroll
        for (int g = 0; g < kGPT; g++) {
          const uint32_t gi = g0 + g * NT;
          valid[g] = gi < groups;
          uint32_t x = valid[g] ? gi : g0;
          for (int b = 0; b < nb; b++) {
            const uint32_t p = seg.bits[b];
            x = ((x >> p) << (p + 1)) | (x & ((1u << p) - 1u));
          }
          gb[g] = x;
#pragma unroll
          for (int k = 0; k < G; k++)
            if (k < (1 << nb)) v[g][k] = sm[swz<Real>(dep(x, k))];
        }
        for (int o = seg.op_begin; o < seg.op_end; o++) {
          if (!ton[o]) continue;
          const SmOp op = sops[o];
          const A* M = smat[o];
          switch (op.code) {
#define MLB_P(kind, rt, c)                                                                       \
  case code_pair(kind, rt, c):                                                                   \
    if constexpr (RB > rt) op_pair<A, G, RB, rt, kind, (bool)c, kGPT>(v, gb, dep, op, M);         \
    break;
#define MLB_PK(kind) MLB_P(kind, 0, 0) MLB_P(kind, 0, 1) MLB_P(kind, 1, 0) MLB_P(kind, 1, 1) \
                     MLB_P(kind, 2, 0) MLB_P(kind, 2, 1) MLB_P(kind, 3, 0) MLB_P(kind, 3, 1)
            MLB_PK(DOP_1Q_GEN) MLB_PK(DOP_1Q_REAL) MLB_PK(DOP_X)
#define MLB_S(a, b, c)                                                                       \
  case code_swap(a, b, c):                                                                   \
    if constexpr (RB > a && RB > b && a != b) op_swap<A, G, RB, a, b, (bool)c, kGPT>(v, gb, dep, op); \
    break;
#define MLB_SS(a, b) MLB_S(a, b, 0) MLB_S(a, b, 1)
            MLB_SS(0, 1) MLB_SS(0, 2) MLB_SS(0, 3) MLB_SS(1, 0) MLB_SS(1, 2) MLB_SS(1, 3)
            MLB_SS(2, 0) MLB_SS(2, 1) MLB_SS(2, 3) MLB_SS(3, 0) MLB_SS(3, 1) MLB_SS(3, 2)
            case code_diag(0, 0): op_diag<A, G, RB, false, false, kGPT>(v, gb, dep, op, M, tkey[o]); break;
            case code_diag(0, 1): op_diag<A, G, RB, false, true, kGPT>(v, gb, dep, op, M, tkey[o]); break;
            case code_diag(1, 0): op_diag<A, G, RB, true, false, kGPT>(v, gb, dep, op, M, tkey[o]); break;
            case code_diag(1, 1): op_diag<A, G, RB, true, false, kGPT>(v, gb, dep, op, M, tkey[o]); break;
#undef MLB_P
#undef MLB_PK
#undef MLB_S
#undef MLB_SS
          }
        }
#pragma unroll
        for (int g = 0; g < kGPT; g++) {
          if (!valid[g]) continue;
#pragma unroll
          for (int k = 0; k < G; k++)
            if (k < (1 << nb)) sm[swz<Real>(dep(gb[g], k))] = v[g][k];
        }
      }
      __syncthreads();
      }  // !DENSE
    }

    // shared -> HBM (streaming stores: the state is far larger than L2), and
    // the next tile's loads into the slots just read
    if (full) {
      constexpr int PER = (1 << TB) / NT;
      const uint64_t next = tile + gridDim.x;
      prefetched = next < pass.num_tiles;
      const uint64_t next_base = prefetched ? pdep64(next, pass.tile_free_mask) : 0;
#pragma unroll 8
      for (int j = 0; j < PER; j++) {
        const uint32_t e = threadIdx.x + j * NT;
        const uint32_t slot = swz<Real>(e);
        const uint64_t off = row_of(e, j) | (e & lmask_low);
        const A v = sm[slot];
        __stcs(&amp[tile_base | off], v);  // consumes v: the slot has been read
        if (prefetched) {
          if constexpr (sizeof(A) == 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sm_base + slot * 16u),
                         "l"(&amp[next_base | off])
                         : "memory");
          else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sm_base + slot * 8u),
                         "l"(&amp[next_base | off])
                         : "memory");
        }
      }
      if (prefetched) asm volatile("cp.async.commit_group;\n" ::: "memory");
    } else {
      for (uint32_t e = threadIdx.x; e < tile_amps; e += NT) {
        const uint64_t gidx = tile_base | rowoff[e >> L] | (e & lmask_low);
        amp[gidx] = sm[swz<Real>(e)];
      }
    }
    __syncthreads();
  }
}

// The shared-memory opt-in is a per-device function attribute; set it once
// per device (threads may race here, and setting it twice is harmless).
template <typename Real>
void prepare_tile_t() {
  using A = typename Cplx<Real>::T;
  static std::atomic<uint64_t> attr_set_mask{0};
  const size_t max_smem = sizeof(A) << TileCfg<Real>::TB;
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set_mask.load(std::memory_order_acquire) & bit)) {
    cudaFuncSetAttribute(k_tile<Real, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    if constexpr (sizeof(Real) == 8)
      cudaFuncSetAttribute(k_tile<Real, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    attr_set_mask.fetch_or(bit, std::memory_order_release);
  }
}

template <typename Real, bool DENSE>
int launch_tile_t(void* amp, const DevPass& pass, const DevSegment* d_segs, const DevOp* d_ops,
                  const DenseSegDev* d_dsegs, const double* d_frags, int num_sms, cudaStream_t stream) {
  using A = typename Cplx<Real>::T;
  constexpr int NT = TileCfg<Real>::NT;
  const size_t smem = sizeof(A) << (pass.L + pass.H);
  prepare_tile_t<Real>();
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile<Real, DENSE>, NT, smem);
  if (per_sm < 1) per_sm = 1;
  uint64_t grid = (uint64_t)num_sms * per_sm;
  if (grid > pass.num_tiles) grid = pass.num_tiles;
  k_tile<Real, DENSE><<<(unsigned)grid, NT, smem, stream>>>(reinterpret_cast<A*>(amp), pass, d_segs, d_ops,
                                                            d_dsegs, d_frags);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

// FP64 tensor-core throughput probe: 8 independent accumulator chains per
// warp, as a dense segment runs them, with the operands in registers; the
// only memory access is one store per thread at the end.
__global__ void __launch_bounds__(256) k_dmma_probe(double* __restrict__ out, int iters, double a0, double b0) {
  double d[8][2];
#pragma unroll
  for (int i = 0; i < 8; i++) d[i][0] = d[i][1] = 0.0;
  const double a = a0 + 1e-9 * threadIdx.x, b = b0;
#pragma unroll 1
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int i = 0; i < 8; i++) dmma_f64(d[i][0], d[i][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += d[i][0] + d[i][1];
  out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

int measure_fp64_tensor_peak(int num_sms, double* tflops) {
  constexpr int kThreads = 256, kIters = 4096, kRuns = 4;
  const int grid = num_sms * 2;  // 16 warps per SM
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * (size_t)grid * kThreads) != cudaSuccess) return MLB_ERR_OUT_OF_MEMORY;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 0.0f;
  int rc = MLB_OK;
  for (int r = 0; r < kRuns && rc == MLB_OK; r++) {  // run 0 warms up
    cudaEventRecord(e0);
    k_dmma_probe<<<grid, kThreads>>>(out, kIters, 1e-3, 1e-3);
    count_launch();
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
      rc = MLB_ERR_DRIVER;
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && (best == 0.0f || ms < best)) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (rc != MLB_OK) return rc;
  // one m8n8k4 mma = 8 x 8 x 4 multiply-adds per warp
  const double flops = 2.0 * 256.0 * 8.0 * kIters * (double)grid * (kThreads / 32);
  *tflops = flops / (best * 1e-3) / 1e12;
  return MLB_OK;
}

void prepare_tile_launch(int dtype) {
  if (dtype == MLB_C128) prepare_tile_t<double>();
  else prepare_tile_t<float>();
}

int launch_tile_pass(int dtype, void* amp, const DevPass& pass, const DevSegment* d_segs,
                     const DevOp* d_ops, const DenseSegDev* d_dsegs, const double* d_frags, int num_sms,
                     cudaStream_t stream, bool all_dense) {
  if (pass.num_segments < 1 || pass.num_segments > kMaxPassSegs) return MLB_ERR_INVALID_ARG;
  // row table size: a tile of a state larger than one tile has the dtype's low bits
  const int TB = dtype == MLB_C128 ? TileCfg<double>::TB : TileCfg<float>::TB;
  const int LOW = dtype == MLB_C128 ? TileCfg<double>::LOW : TileCfg<float>::LOW;
  if (pass.L + pass.H > TB || (pass.H > 0 && pass.L != LOW)) return MLB_ERR_INVALID_ARG;
  if (dtype == MLB_C128) {
    if (all_dense) return launch_tile_t<double, true>(amp, pass, d_segs, d_ops, d_dsegs, d_frags, num_sms, stream);
    return launch_tile_t<double, false>(amp, pass, d_segs, d_ops, d_dsegs, d_frags, num_sms, stream);
  }
  return launch_tile_t<float, false>(amp, pass, d_segs, d_ops, nullptr, nullptr, num_sms, stream);
}

}  // namespace mlb
