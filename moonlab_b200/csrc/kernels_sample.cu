// kernels_sample.cu -- the reference's sequential FP64 sums, reproduced
// exactly on the GPU, and sampling / collapse built on them.
//
// The reference draws outcomes from a left-to-right running sum
//     s_i = fl(s_{i-1} + p_i),  p_i = fl(cabs(a_i) * cabs(a_i))
// (measurement_sample, measurement.c:551-601; measurement_all_qubits,
// :263-307; qgtl shots, moonlab_qgtl_backend.c:218-243) and decides
// single-qubit outcomes from the same kind of sum over half of the indices
// (measurement_probability_one, measurement.c:73; quantum_measure,
// gates.c:1117-1241).  A parallel sum rounds differently, so an outcome
// near a CDF boundary could differ.  This file reproduces s_i exactly:
//
//  * p_i: hypot_glibc.cuh reproduces glibc's cabs bit for bit.
//  * Within one binade [2^e, 2^(e+1)) every representable s is a multiple of
//    g = ulp(2^e), so fl(s + p) = s + g * k with k = p/g rounded to nearest,
//    ties to the k that makes (s/g + k) even.  Only the tie case depends on
//    s, and only through the parity of s/g.  A chunk of elements therefore
//    maps (N = s/g, parity) -> (N + K[parity], parity') with two integer
//    increments, computed in parallel as an ordered reduction of 2-entry
//    transfer tables (phase C).  The tables compose associatively, so the
//    chunks are chained from the exact running value by an ordered scan of
//    their tables (phase D); a chunk whose sum leaves the binade, whose
//    predicted binade was wrong, or which starts at s = 0 with a nonzero
//    contribution is summed element by element instead.  The binade of each
//    chunk's start is predicted from an ordinary parallel prefix of chunk
//    totals (phases A, B).
//  * Sampling (phase E): one warp per uniform finds the chunk whose exact
//    end value first passes u and replays that chunk's adds in hardware
//    FP64 (IEEE round to nearest, hence bit-identical).
//
// A filter (index & fmask) == fval restricts the sum to a subspace: elements
// outside it contribute p = 0, and fl(s + 0) = s, so the filtered running
// sum equals the reference's sum over the subspace in index order.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "hypot_glibc.cuh"
#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

constexpr int kCB = 12;             // chunk = 2^12 elements (33 KiB of p in shared memory)
constexpr int kCT = 256;            // threads per CTA
constexpr int kPer = (1 << kCB) / kCT;  // 32 contiguous elements per thread
constexpr long long kTwo53 = 1ll << 53;
constexpr int kDPer = 8;                // phase D: chunks per thread in one scan
constexpr int kDBatch = kCT * kDPer;     // phase D: 2048 chunks per scan
constexpr int kNoBinade = -0x40000000;   // matches no candidate binade
constexpr int kZeroChunk = 0x7fffffff;   // Xfer::e[0] of a chunk that adds 0 for every s

struct alignas(16) Xfer {  // per chunk: transfer tables for two candidate binades (3 x 16 bytes)
  int32_t e[2];        // binade exponents (INT32_MIN: unused; e[0] == kZeroChunk: adds 0 for every s)
  int32_t P;           // exit parities: bit 2 cand + entry parity
  int32_t pad;
  long long K[2][2];   // [candidate][entry parity] increments, saturated at 2^53
};

struct SeqScratch {
  double* chunk_tot;   // [nc] plain FP64 chunk totals (phase A)
  double* chunk_pre;   // [nc] exclusive prefix of chunk totals (phase B)
  Xfer* xfer;          // [nc]
  double* s_in;        // [nc + 1] exact running value before chunk c; s_in[nc] = total
  long long* lastnz;   // [1] largest index with p > 0 (within the filter), -1 if none
  double* uni;         // [num] uniforms (sampling)
  unsigned long long* outc;  // [num] outcomes (sampling)
};

template <typename Real>
__device__ __forceinline__ double elem_p(const typename Cplx<Real>::T* __restrict__ amp, uint64_t i,
                                         uint64_t fmask, uint64_t fval) {
  if ((i & fmask) != fval) return 0.0;
  const auto a = amp[i];
  return glibc_prob((double)a.x, (double)a.y);
}

// Two accumulation contracts, as the reference's Release build compiles its
// loops: SEPARATE  s = fl(s + fl(h*h))   (measurement_sample,
// measurement_all_qubits, quantum_measure) and FUSED  s = fma(h, h, s)
// (measurement_probability_one, measurement_single_qubit).  The per-element
// value kept in shared memory is p = fl(h*h) for SEPARATE and h for FUSED.
template <typename Real, bool FUSED>
__device__ __forceinline__ double elem_val(const typename Cplx<Real>::T* __restrict__ amp, uint64_t i,
                                           uint64_t fmask, uint64_t fval) {
  if ((i & fmask) != fval) return 0.0;
  const auto a = amp[i];
  const double h = glibc_cabs((double)a.x, (double)a.y);
  return FUSED ? h : __dmul_rn(h, h);
}
template <bool FUSED>
__device__ __forceinline__ double elem_add(double s, double v) {
  return FUSED ? __fma_rn(v, v, s) : __dadd_rn(s, v);
}

// binade exponent of s > 0 (s in [2^e, 2^(e+1))) and its grid spacing
__device__ __forceinline__ int binade_of(double s) {
  const unsigned long long b = __double_as_longlong(s);
  const int ex = (int)((b >> 52) & 0x7ff);
  if (ex == 0) return -1023;  // subnormal: grid 2^-1074
  return ex - 1023;
}
__device__ __forceinline__ double grid_of(int e) {
  const int ge = e - 52;
  return ge < -1074 ? 0x1p-1074 : ldexp(1.0, ge);
}

// Load a chunk's p values into shared memory (coalesced) -- p[j] for j in
// [0, len), padded by one slot per 32 to spread banks for the contiguous
// per-thread reads that follow.
template <typename Real, bool FUSED>
__device__ __forceinline__ void load_chunk_p(const typename Cplx<Real>::T* __restrict__ amp,
                                             uint64_t base, uint32_t len, uint64_t fmask,
                                             uint64_t fval, double* sp) {
  for (uint32_t j = threadIdx.x; j < len; j += kCT)
    sp[j + (j >> 5)] = elem_val<Real, FUSED>(amp, base + j, fmask, fval);
}

// Phase A's per-element value: |a|^2 as x^2 + y^2, which is within a few
// ulp of the reference's fl(cabs(a)^2).  The totals only predict each
// chunk's binade (phase C allows ~10^6 ulp for it, and a wrong prediction
// only sends the chunk to the exact replay), so glibc's algorithm is needed
// only where the approximation could disagree on p > 0 (the last nonzero
// index must be exact): below 2^-1000, and for inf / nan.
template <typename Real, bool FUSED>
__device__ __forceinline__ double elem_p_approx(const typename Cplx<Real>::T* __restrict__ amp, uint64_t i,
                                                uint64_t fmask, uint64_t fval) {
  if ((i & fmask) != fval) return 0.0;
  const auto a = amp[i];
  const double x = (double)a.x, y = (double)a.y;
  const double pa = fma(x, x, y * y);
  if (pa >= 0x1p-1000 && pa <= 0x1.fffffffffffffp+1023) return pa;
  const double h = glibc_cabs(x, y);
  return FUSED ? h * h : __dmul_rn(h, h);
}

// Phase C's per-element value, on the candidate grids of the chunk
// (inv_g = 1/g; 0: no such candidate).  Element transfer (elem_fn) uses only
// k = (contribution)/g rounded to nearest.  x^2 + y^2 (one fma) is within
// 2^-50 of the contribution -- SEPARATE's fl(cabs(a)^2) and FUSED's exact
// cabs(a)^2 -- as hypot is within one ulp and each side rounds once more
// (2^-51 measured against glibc on 2*10^8 inputs).  So where x^2 + y^2,
// scaled to a grid, lies more than 2^-48 of itself away from a half-integer
// (and below 2^52), both round to the same k, no tie occurs, and elem_fn
// gives the same transfer; elsewhere glibc's algorithm is used.  The value
// kept is p for SEPARATE; for FUSED it is h, or -(x^2 + y^2) on the fast path.
__device__ __forceinline__ bool grid_safe(double pa, double inv_g) {
  const double q = pa * inv_g;  // exact scaling by a power of two
  if (!(q < 0x1p52)) return false;
  const double fr = q - floor(q);
  return fabs(fr - 0.5) > q * 0x1p-48;
}
template <typename Real, bool FUSED>
__device__ __forceinline__ double elem_p_on_grids(const typename Cplx<Real>::T* __restrict__ amp, uint64_t i,
                                                  uint64_t fmask, uint64_t fval, double ig0, double ig1) {
  if ((i & fmask) != fval) return 0.0;
  const auto a = amp[i];
  const double x = (double)a.x, y = (double)a.y;
  const double pa = fma(x, x, y * y);
  if (pa >= 0x1p-1000 && grid_safe(pa, ig0) && grid_safe(pa, ig1)) return FUSED ? -pa : pa;
  const double h = glibc_cabs(x, y);
  return FUSED ? h : __dmul_rn(h, h);
}

// Phase A: chunk totals (plain FP64, in a fixed order) and the last nonzero
// index.  One warp per chunk, lane-strided coalesced loads; the order of the
// additions does not matter here, so there is no staging and no barrier.
template <typename Real, bool FUSED>
__global__ void __launch_bounds__(kCT) k_seq_a(const typename Cplx<Real>::T* __restrict__ amp,
                                               uint64_t nc, uint32_t clen, uint64_t fmask,
                                               uint64_t fval, double* __restrict__ chunk_tot,
                                               long long* __restrict__ lastnz) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (kCT / 32);
  long long lnz_all = -1;
  for (uint64_t c = (uint64_t)blockIdx.x * (kCT / 32) + (threadIdx.x >> 5); c < nc; c += nwarps) {
    const uint64_t base = c * clen;
    double t = 0.0;
    long long lnz = -1;
#pragma unroll 8
    for (uint32_t j = lane; j < clen; j += 32) {
      const double p = elem_p_approx<Real, FUSED>(amp, base + j, fmask, fval);
      t += p;
      if (p > 0.0) lnz = (long long)(base + j);
    }
    for (int o = 16; o > 0; o >>= 1) {
      t += __shfl_down_sync(0xffffffffu, t, o);
      lnz = max(lnz, __shfl_down_sync(0xffffffffu, lnz, o));
    }
    if (lane == 0) chunk_tot[c] = t;
    lnz_all = max(lnz_all, lnz);
  }
  if (lane == 0 && lnz_all >= 0) atomicMax(lastnz, lnz_all);
}

// Phase B: exclusive prefix of chunk totals (one CTA; fixed order).
__global__ void __launch_bounds__(1024) k_seq_b(const double* __restrict__ tot, uint64_t nc,
                                                double* __restrict__ pre) {
  __shared__ double part[1024];
  const uint64_t per = (nc + 1023) / 1024;
  const uint64_t lo = threadIdx.x * per, hi = min(nc, lo + per);
  double s = 0.0;
  for (uint64_t c = lo; c < hi; c++) s += tot[c];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double run = 0.0;
    for (int i = 0; i < 1024; i++) { const double v = part[i]; part[i] = run; run += v; }
  }
  __syncthreads();
  double run = part[threadIdx.x];
  for (uint64_t c = lo; c < hi; c++) { pre[c] = run; run += tot[c]; }
}

struct Fn {  // transfer table: entry parity -> (increment, exit parity)
  long long K0, K1;
  int P0, P1;
};
__device__ __forceinline__ long long sat_add(long long a, long long b) {
  const long long r = a + b;
  return r > kTwo53 ? kTwo53 : r;
}
__device__ __forceinline__ Fn compose(const Fn& f, const Fn& g) {  // g after f
  Fn r;
  r.K0 = sat_add(f.K0, f.P0 ? g.K1 : g.K0);
  r.P0 = f.P0 ? g.P1 : g.P0;
  r.K1 = sat_add(f.K1, f.P1 ? g.K1 : g.K0);
  r.P1 = f.P1 ? g.P1 : g.P0;
  return r;
}

// Element transfer on grid g (inv_g = 1/g, an exact power of two).  The
// element adds the exact real v = hi + lo to the running sum: SEPARATE has
// v = p (lo = 0); FUSED has v = h*h exactly, hi = fl(h*h), lo = fma(h,h,-hi).
// With q = v/g = qh + ql (both exact scalings), fl = floor(qh) and
// r = qh - fl (exact), the nearest integer to q is fl + 1 when r > 1/2 or
// (r == 1/2 and ql > 0), fl when r < 1/2 or (r == 1/2 and ql < 0), and a tie
// only when r == 1/2 and ql == 0: |ql| <= ulp(qh)/2 and r lies on qh's
// grid, so ql can only decide the case r == 1/2.  FUSED with v < 0: -v is
// the contribution itself, x^2 + y^2 at a position where it rounds to the
// same increment as h*h (elem_p_on_grids), with lo = 0.
template <bool FUSED>
__device__ __forceinline__ Fn elem_fn(double v, double inv_g) {
  Fn f;
  if (v == 0.0) { f.K0 = 0; f.K1 = 0; f.P0 = 0; f.P1 = 1; return f; }
  double hi = v, lo = 0.0;
  if (FUSED && v < 0.0) {
    hi = -v;
  } else if (FUSED) {
    hi = __dmul_rn(v, v);
    lo = __fma_rn(v, v, -hi);
    if (hi == 0.0) { f.K0 = 0; f.K1 = 0; f.P0 = 0; f.P1 = 1; return f; }
  }
  const double q = hi * inv_g;  // exact scaling by a power of two
  if (!(q < 0x1p53)) { f.K0 = kTwo53; f.K1 = kTwo53; f.P0 = 0; f.P1 = 0; return f; }
  const double ql = lo * inv_g;
  const double fl = floor(q);
  const double fr = q - fl;   // exact
  const long long k = (long long)fl;
  const bool up = fr > 0.5 || (fr == 0.5 && ql > 0.0);
  const bool down = fr < 0.5 || (fr == 0.5 && ql < 0.0);
  if (up || down) {
    const long long kk = k + (up ? 1 : 0);
    f.K0 = kk; f.K1 = kk;
    f.P0 = (int)(kk & 1);
    f.P1 = (int)((kk + 1) & 1);
    return f;
  }
  // tie: choose the increment that makes N + increment even
  const long long k0 = k + ((0 + k) & 1);   // entry parity 0
  const long long k1 = k + ((1 + k) & 1);   // entry parity 1
  f.K0 = k0; f.K1 = k1; f.P0 = 0; f.P1 = 0;
  return f;
}

// Phase C: transfer tables for the two candidate binades of each chunk.
template <typename Real, bool FUSED>
__global__ void __launch_bounds__(kCT) k_seq_c(const typename Cplx<Real>::T* __restrict__ amp,
                                               uint64_t nc, uint32_t clen, uint64_t fmask,
                                               uint64_t fval, const double* __restrict__ ctot,
                                               const double* __restrict__ pre,
                                               Xfer* __restrict__ xfer) {
  __shared__ double sp[(1 << kCB) + (1 << kCB) / 32];
  __shared__ Fn red[kCT / 32][2];
  const double u = 0x1p-53;
  for (uint64_t c = blockIdx.x; c < nc; c += gridDim.x) {
    const uint64_t base = c * clen;
    // candidate binades of the running value at the chunk start: the
    // prefix estimate +- a bound on both its error and the reference's.
    const double S = pre[c];
    int ecand[2] = {INT32_MIN, INT32_MIN};
    if (S > 0.0) {
      const double rel = ((double)base * 4.0 + 1.0e6) * u;
      const int elo = binade_of(S * (1.0 - rel)), ehi = binade_of(S * (1.0 + rel));
      ecand[0] = elo;
      ecand[1] = (ehi == elo) ? INT32_MIN : ehi;
      if (ehi - elo > 1) { ecand[0] = INT32_MIN; ecand[1] = INT32_MIN; }  // too uncertain
    }
    const double ig0 = ecand[0] != INT32_MIN ? 1.0 / grid_of(ecand[0]) : 0.0;  // exact: powers of two
    const double ig1 = ecand[1] != INT32_MIN ? 1.0 / grid_of(ecand[1]) : 0.0;
    for (uint32_t j = threadIdx.x; j < clen; j += kCT)
      sp[j + (j >> 5)] = elem_p_on_grids<Real, FUSED>(amp, base + j, fmask, fval, ig0, ig1);
    __syncthreads();
    for (int cand = 0; cand < 2; cand++) {
      Fn acc = {0, 0, 0, 1};  // identity
      if (ecand[cand] == INT32_MIN) {  // no such candidate (uniform over the CTA)
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][cand] = acc;
        continue;
      }
      const double inv_g = cand ? ig1 : ig0;
      for (int k = 0; k < kPer; k++) {
        const uint32_t j = threadIdx.x * kPer + k;
        if (j < clen) acc = compose(acc, elem_fn<FUSED>(sp[j + (j >> 5)], inv_g));
      }
      // ordered warp reduction: lane l combines [l, l+o) with [l+o, l+2o)
      for (int o = 1; o < 32; o <<= 1) {
        Fn other;
        other.K0 = __shfl_down_sync(0xffffffffu, acc.K0, o);
        other.K1 = __shfl_down_sync(0xffffffffu, acc.K1, o);
        other.P0 = __shfl_down_sync(0xffffffffu, acc.P0, o);
        other.P1 = __shfl_down_sync(0xffffffffu, acc.P1, o);
        if ((threadIdx.x & 31) + o < 32 && ((threadIdx.x & (2 * o - 1)) == 0)) acc = compose(acc, other);
      }
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][cand] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      Xfer x;
      int pbits = 0;
      for (int cand = 0; cand < 2; cand++) {
        Fn a = {0, 0, 0, 1};
        for (int w = 0; w < kCT / 32; w++) a = compose(a, red[w][cand]);
        x.e[cand] = ecand[cand];
        x.K[cand][0] = a.K0; x.K[cand][1] = a.K1;
        pbits |= (a.P0 | (a.P1 << 1)) << (2 * cand);
      }
      x.P = pbits;
      x.pad = 0;
      // Every contribution is 0 exactly when the plain total is 0 (the
      // values are >= 0; for FUSED, h*h rounds to 0 only below half the
      // smallest subnormal, which then also leaves any s unchanged).
      if (ctot[c] == 0.0) x.e[0] = kZeroChunk;
      xfer[c] = x;
    }
    __syncthreads();
  }
}

// Phase D: the exact running value at every chunk start, one CTA.  Transfer
// tables compose associatively, so the chunks are taken kDBatch at a time
// from the exact value b at the batch start: each thread composes the tables
// of kDPer consecutive chunks for b's binade, the CTA scans those
// compositions in order, and each thread walks its chunks again from its
// exclusive prefix, writing s_in.  Increments are nonnegative, so the
// running value only grows: the first chunk whose end leaves the binade, or
// which has no table for it, is the first failure.  The values up to its
// start are exact; that chunk is replayed element by element and the next
// batch starts after it.  A chunk whose every contribution is 0 is the
// identity for any s, so runs of such chunks pass even at s = 0.

// Chunk c's map for binade e: three independent 16-byte loads, then a select.
__device__ __forceinline__ Fn chunk_fn(const Xfer* __restrict__ xfer, uint64_t c, int e) {
  const int4 h = __ldg(reinterpret_cast<const int4*>(xfer + c));
  const longlong2 k0 = __ldg(reinterpret_cast<const longlong2*>(xfer + c) + 1);
  const longlong2 k1 = __ldg(reinterpret_cast<const longlong2*>(xfer + c) + 2);
  if (h.x == kZeroChunk) return Fn{0, 0, 0, 1};
  const int cand = (h.x == e) ? 0 : (h.y == e) ? 1 : -1;
  if (cand < 0) return Fn{kTwo53, kTwo53, 0, 1};
  const int pb = h.z >> (2 * cand);
  return cand == 0 ? Fn{k0.x, k0.y, pb & 1, (pb >> 1) & 1} : Fn{k1.x, k1.y, pb & 1, (pb >> 1) & 1};
}
__device__ __forceinline__ Fn shfl_up_fn(const Fn& f, int o) {
  Fn r;
  r.K0 = __shfl_up_sync(0xffffffffu, f.K0, o);
  r.K1 = __shfl_up_sync(0xffffffffu, f.K1, o);
  r.P0 = __shfl_up_sync(0xffffffffu, f.P0, o);
  r.P1 = __shfl_up_sync(0xffffffffu, f.P1, o);
  return r;
}

template <typename Real, bool FUSED>
__global__ void __launch_bounds__(kCT) k_seq_d(const typename Cplx<Real>::T* __restrict__ amp,
                                               uint64_t nc, uint32_t clen, uint64_t fmask,
                                               uint64_t fval, const Xfer* __restrict__ xfer,
                                               double* __restrict__ s_in) {
  __shared__ double sp[(1 << kCB) + (1 << kCB) / 32];
  __shared__ Fn wtot[kCT / 32];
  __shared__ unsigned int s_fail;
  __shared__ double s_run;
  const Fn ident = {0, 0, 0, 1};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long* s_bits = (unsigned long long*)s_in;
  uint64_t c = 0;
  unsigned long long b = 0;  // bit pattern of the exact running value (s >= 0)
  while (c < nc) {
    // s = N g in its binade; (N + K) g has the bit pattern b + K while
    // N + K < 2^53, i.e. while b + K stays below `limit` (for a subnormal s
    // the grid 2^-1074 also covers the lowest normal binade).
    const int ex = (int)(b >> 52);
    int e;
    unsigned long long limit;
    if (b == 0ull) { e = kNoBinade; limit = 1; }                // only all-zero chunks pass
    else if (ex == 0x7ff) { e = kNoBinade; limit = 0; }         // inf / nan: replayed
    else {
      e = ex ? ex - 1023 : -1023;
      limit = ex ? ((unsigned long long)(ex + 1) << 52) : (2ull << 52);
    }
    const int pb = (int)(b & 1ull);
    const uint64_t c0 = c;
    const uint64_t lo = c0 + (uint64_t)threadIdx.x * kDPer;
    // this thread's chunk maps, loaded together and kept for both walks
    Fn f[kDPer];
#pragma unroll
    for (int k = 0; k < kDPer; k++) f[k] = lo + k < nc ? chunk_fn(xfer, lo + k, e) : ident;
    Fn acc = ident;
#pragma unroll
    for (int k = 0; k < kDPer; k++) acc = compose(acc, f[k]);
    for (int o = 1; o < 32; o <<= 1) {  // inclusive scan over the warp, in order
      const Fn other = shfl_up_fn(acc, o);
      if (lane >= o) acc = compose(other, acc);
    }
    if (lane == 31) wtot[warp] = acc;
    if (threadIdx.x == 0) s_fail = 0xffffffffu;
    __syncthreads();
    Fn pre = ident;
    for (int w = 0; w < warp; w++) pre = compose(pre, wtot[w]);
    const Fn lane_ex = shfl_up_fn(acc, 1);
    if (lane > 0) pre = compose(pre, lane_ex);
    // walk this thread's chunks from the exact entry state (increment, parity)
    long long kin = pb ? pre.K1 : pre.K0;
    int par = pb ? pre.P1 : pre.P0;
    bool walking = true;
#pragma unroll
    for (int k = 0; k < kDPer; k++) {
      const uint64_t i = lo + k;
      if (walking && i < nc) {
        s_bits[i] = b + (unsigned long long)kin;
        kin = sat_add(kin, par ? f[k].K1 : f[k].K0);
        par = par ? f[k].P1 : f[k].P0;
        if (b + (unsigned long long)kin >= limit) {
          atomicMin(&s_fail, (unsigned int)(i - c0));
          walking = false;
        }
      }
    }
    __syncthreads();
    const unsigned int fail = s_fail;
    if (fail == 0xffffffffu) {
      Fn tot = ident;
      for (int w = 0; w < kCT / 32; w++) tot = compose(tot, wtot[w]);
      b += (unsigned long long)(pb ? tot.K1 : tot.K0);
      c = min(nc, c0 + (uint64_t)kDBatch);
      __syncthreads();  // wtot is rewritten by the next batch
      continue;
    }
    // element-by-element replay of the first failing chunk from its exact start
    c = c0 + fail;
    load_chunk_p<Real, FUSED>(amp, c * clen, clen, fmask, fval, sp);
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = __longlong_as_double((long long)s_bits[c]);
#pragma unroll 8
      for (uint32_t j = 0; j < clen; j++) s = elem_add<FUSED>(s, sp[j + (j >> 5)]);
      s_run = s;
    }
    __syncthreads();
    b = (unsigned long long)__double_as_longlong(s_run);
    c++;
    __syncthreads();
  }
  if (threadIdx.x == 0) s_bits[nc] = b;
}

// Phase E: one warp per uniform.
template <typename Real>
__global__ void __launch_bounds__(kCT) k_seq_e(const typename Cplx<Real>::T* __restrict__ amp,
                                               uint64_t nc, uint32_t clen, uint64_t dim, int rule,
                                               const double* __restrict__ s_in,
                                               const long long* __restrict__ lastnz,
                                               const double* __restrict__ uni, uint64_t num,
                                               unsigned long long* __restrict__ out) {
  const uint64_t w = ((uint64_t)blockIdx.x * kCT + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= num) return;
  const double u = uni[w];
  // first chunk c whose end value s_in[c+1] passes u (>= for rule 0, > for rule 1)
  uint64_t lo = 0, hi = nc;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    const double end = s_in[mid + 1];
    const bool pass = rule == 0 ? (end >= u) : (end > u);
    if (pass) hi = mid; else lo = mid + 1;
  }
  if (lo >= nc) {
    if (lane == 0) {
      if (rule == 0) out[w] = dim - 1;
      else out[w] = (unsigned long long)(lastnz[0] >= 0 ? lastnz[0] : 0);
    }
    return;
  }
  const uint64_t c = lo, base = c * clen;
  double s = s_in[c];
  unsigned long long found = ~0ull;
  for (uint32_t j0 = 0; j0 < clen && found == ~0ull; j0 += 32) {
    const uint32_t j = j0 + lane;
    const double p = j < clen ? elem_p<Real>(amp, base + j, 0, 0) : 0.0;
    // lane 0 replays the 32 adds in order
    for (int l = 0; l < 32; l++) {
      const double pl = __shfl_sync(0xffffffffu, p, l);
      if (lane == 0 && found == ~0ull && j0 + l < clen) {
        s = __dadd_rn(s, pl);
        const bool hit = rule == 0 ? (s >= u) : (u < s);
        if (hit) found = base + j0 + l;
      }
    }
    found = __shfl_sync(0xffffffffu, found, 0);
  }
  if (lane == 0) {
    // The chunk end passes u, so the replay must hit inside it.
    out[w] = found != ~0ull ? found : (rule == 0 ? dim - 1 : (unsigned long long)base + clen - 1);
  }
}

struct Cache {
  int device = -1;
  size_t bytes = 0;
  void* mem = nullptr;
};
thread_local Cache g_cache;

SeqScratch get_scratch(uint64_t nc, size_t num, cudaStream_t stream) {
  const size_t need = sizeof(double) * nc * 2 + sizeof(Xfer) * nc + sizeof(double) * (nc + 1) +
                      sizeof(long long) + sizeof(double) * num + sizeof(uint64_t) * num + 256 * 7;
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_cache.mem == nullptr || g_cache.bytes < need || g_cache.device != dev) {
    if (g_cache.mem) {
      cudaStreamSynchronize(stream);
      cudaFree(g_cache.mem);
    }
    g_cache.mem = nullptr;
    if (cudaMalloc(&g_cache.mem, need) != cudaSuccess) {
      g_cache = Cache{};
      return SeqScratch{};
    }
    g_cache.bytes = need;
    g_cache.device = dev;
  }
  char* p = (char*)g_cache.mem;
  auto take = [&](size_t b) { char* r = p; p += (b + 255) & ~(size_t)255; return (void*)r; };
  SeqScratch s;
  s.chunk_tot = (double*)take(sizeof(double) * nc);
  s.chunk_pre = (double*)take(sizeof(double) * nc);
  s.xfer = (Xfer*)take(sizeof(Xfer) * nc);
  s.s_in = (double*)take(sizeof(double) * (nc + 1));
  s.lastnz = (long long*)take(sizeof(long long));
  s.uni = (double*)take(sizeof(double) * num);
  s.outc = (unsigned long long*)take(sizeof(uint64_t) * num);
  return s;
}

// Run phases A-D; on return s_in[0..nc] are the exact running values.
template <typename Real, bool FUSED>
int seq_prepare(const void* amp_v, int n, uint64_t fmask, uint64_t fval, size_t num, int num_sms,
                cudaStream_t stream, SeqScratch& sc, uint64_t& nc, uint32_t& clen) {
  using A = typename Cplx<Real>::T;
  const A* amp = (const A*)amp_v;
  const uint64_t dim = 1ull << n;
  clen = n >= kCB ? (1u << kCB) : (uint32_t)dim;
  nc = dim / clen;
  sc = get_scratch(nc, num, stream);
  if (!sc.chunk_tot) return MLB_ERR_OUT_OF_MEMORY;
  const long long neg1 = -1;
  cudaMemcpyAsync(sc.lastnz, &neg1, sizeof(neg1), cudaMemcpyHostToDevice, stream);
  // phase A: one warp per chunk, 5 CTAs per SM (its 48 registers allow 5);
  // phase C: one CTA per chunk, 6 CTAs per SM (its shared memory allows 6)
  const int grid_a = (int)std::min<uint64_t>((nc + kCT / 32 - 1) / (kCT / 32), (uint64_t)num_sms * 5);
  const int grid = (int)std::min<uint64_t>(nc, (uint64_t)num_sms * 6);
  k_seq_a<Real, FUSED><<<grid_a, kCT, 0, stream>>>(amp, nc, clen, fmask, fval, sc.chunk_tot, sc.lastnz);
  k_seq_b<<<1, 1024, 0, stream>>>(sc.chunk_tot, nc, sc.chunk_pre);
  k_seq_c<Real, FUSED><<<grid, kCT, 0, stream>>>(amp, nc, clen, fmask, fval, sc.chunk_tot,
                                                 sc.chunk_pre, sc.xfer);
  k_seq_d<Real, FUSED><<<1, kCT, 0, stream>>>(amp, nc, clen, fmask, fval, sc.xfer, sc.s_in);
  count_launch(4);
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

template <typename Real>
int sample_t(const void* amp, int n, int rule, const double* h_u, size_t num, uint64_t* h_out,
             int num_sms, cudaStream_t stream) {
  SeqScratch sc;
  uint64_t nc;
  uint32_t clen;
  int rc = seq_prepare<Real, false>(amp, n, 0, 0, num, num_sms, stream, sc, nc, clen);
  if (rc) return rc;
  if (num == 0) return MLB_OK;
  double* d_u = sc.uni;
  unsigned long long* d_o = sc.outc;
  cudaMemcpyAsync(d_u, h_u, num * sizeof(double), cudaMemcpyHostToDevice, stream);
  const uint64_t threads = num * 32;
  const unsigned grid = (unsigned)((threads + kCT - 1) / kCT);
  k_seq_e<Real><<<grid, kCT, 0, stream>>>((const typename Cplx<Real>::T*)amp, nc, clen, 1ull << n,
                                          rule, sc.s_in, sc.lastnz, d_u, num, d_o);
  count_launch();
  cudaMemcpyAsync(h_out, d_o, num * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream);
  if (cudaStreamSynchronize(stream) != cudaSuccess) return MLB_ERR_DRIVER;
  return MLB_OK;
}

template <typename Real>
int seq_total(const void* amp, int n, uint64_t fmask, uint64_t fval, bool fused, int num_sms,
              cudaStream_t stream, double* total) {
  SeqScratch sc;
  uint64_t nc;
  uint32_t clen;
  int rc = fused ? seq_prepare<Real, true>(amp, n, fmask, fval, 0, num_sms, stream, sc, nc, clen)
                 : seq_prepare<Real, false>(amp, n, fmask, fval, 0, num_sms, stream, sc, nc, clen);
  if (rc) return rc;
  cudaMemcpyAsync(total, sc.s_in + nc, sizeof(double), cudaMemcpyDeviceToHost, stream);
  if (cudaStreamSynchronize(stream) != cudaSuccess) return MLB_ERR_DRIVER;
  return MLB_OK;
}

}  // namespace

int sample_exact(int dtype, const void* amp, int n, int rule, const double* h_uniforms, size_t num,
                 uint64_t* h_out, int num_sms, cudaStream_t stream, char* errbuf, size_t errlen) {
  (void)errbuf;
  (void)errlen;
  if (dtype == MLB_C128) return sample_t<double>(amp, n, rule, h_uniforms, num, h_out, num_sms, stream);
  return sample_t<float>(amp, n, rule, h_uniforms, num, h_out, num_sms, stream);
}

int seq_sum_exact(int dtype, const void* amp, int n, uint64_t fmask, uint64_t fval, bool fused,
                  int num_sms, cudaStream_t stream, double* total) {
  if (dtype == MLB_C128) return seq_total<double>(amp, n, fmask, fval, fused, num_sms, stream, total);
  return seq_total<float>(amp, n, fmask, fval, fused, num_sms, stream, total);
}

}  // namespace mlb
