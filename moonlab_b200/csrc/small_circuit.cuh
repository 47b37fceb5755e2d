// small_circuit.cuh -- device code shared by the small-circuit kernels
// (kernels_small.cu: many circuits per launch; kernels_mailbox.cu: the
// persistent request loop): one op at a time on a state held in shared
// memory by a whole thread block.
#pragma once

#include "kernels_common.cuh"
#include "hypot_glibc.cuh"
#include "mlb_internal.h"

namespace mlb {
namespace small {

constexpr int kST = 256;  // threads per CTA

template <typename A>
__device__ __forceinline__ A cmadd(double mr, double mi, A a, A acc) {
  using R = decltype(a.x);
  acc.x += (R)mr * a.x - (R)mi * a.y;
  acc.y += (R)mr * a.y + (R)mi * a.x;
  return acc;
}
template <typename A>
__device__ __forceinline__ A cscale(double mr, double mi, A a) {
  using R = decltype(a.x);
  A r;
  r.x = (R)mr * a.x - (R)mi * a.y;
  r.y = (R)mr * a.y + (R)mi * a.x;
  return r;
}

// Insert a zero bit at position b.
__device__ __forceinline__ uint32_t ins0(uint32_t x, uint32_t b) {
  return ((x >> b) << (b + 1)) | (x & ((1u << b) - 1u));
}

// One op on the shared-memory state (all threads; the caller synchronises).
template <typename A>
__device__ void apply_op(A* st, uint32_t n, const mlb_op_t& o) {
  const uint32_t dim = 1u << n;
  const uint32_t cm = (uint32_t)o.cmask;
  const double* m = o.m;
  switch (o.kind) {
    case MLB_OP_1Q:
    case MLB_OP_X: {
      const uint32_t t = (uint32_t)o.target, tb = 1u << t;
      for (uint32_t j = threadIdx.x; j < (dim >> 1); j += kST) {
        const uint32_t i0 = ins0(j, t);
        if ((i0 & cm) != cm) continue;
        const A a0 = st[i0], a1 = st[i0 | tb];
        if (o.kind == MLB_OP_X) {
          st[i0] = a1;
          st[i0 | tb] = a0;
        } else {
          st[i0] = cmadd(m[2], m[3], a1, cscale(m[0], m[1], a0));
          st[i0 | tb] = cmadd(m[6], m[7], a1, cscale(m[4], m[5], a0));
        }
      }
      return;
    }
    case MLB_OP_DIAG1: {
      const uint32_t tb = 1u << o.target;
      for (uint32_t i = threadIdx.x; i < dim; i += kST) {
        if ((i & cm) != cm) continue;
        st[i] = (i & tb) ? cscale(m[2], m[3], st[i]) : cscale(m[0], m[1], st[i]);
      }
      return;
    }
    case MLB_OP_PHASE: {
      for (uint32_t i = threadIdx.x; i < dim; i += kST)
        if ((i & cm) == cm) st[i] = cscale(m[0], m[1], st[i]);
      return;
    }
    case MLB_OP_ZZ: {
      const uint32_t b0 = 1u << o.target, b1 = 1u << o.target2;
      for (uint32_t i = threadIdx.x; i < dim; i += kST) {
        if ((i & cm) != cm) continue;
        const bool same = ((i & b0) != 0) == ((i & b1) != 0);
        st[i] = same ? cscale(m[0], m[1], st[i]) : cscale(m[2], m[3], st[i]);
      }
      return;
    }
    case MLB_OP_2Q:
    case MLB_OP_SWAP: {
      const uint32_t t0 = (uint32_t)o.target, t1 = (uint32_t)o.target2;
      const uint32_t lo = t0 < t1 ? t0 : t1, hi = t0 < t1 ? t1 : t0;
      const uint32_t b0 = 1u << t0, b1 = 1u << t1;
      for (uint32_t j = threadIdx.x; j < (dim >> 2); j += kST) {
        const uint32_t i = ins0(ins0(j, lo), hi);
        if ((i & cm) != cm) continue;
        if (o.kind == MLB_OP_SWAP) {
          const A t = st[i | b0];
          st[i | b0] = st[i | b1];
          st[i | b1] = t;
          continue;
        }
        const uint32_t idx[4] = {i, i | b0, i | b1, i | b0 | b1};
        A x[4];
#pragma unroll
        for (int c = 0; c < 4; c++) x[c] = st[idx[c]];
#pragma unroll
        for (int r = 0; r < 4; r++) {
          A acc = cscale(m[(r * 4) * 2], m[(r * 4) * 2 + 1], x[0]);
#pragma unroll
          for (int c = 1; c < 4; c++) acc = cmadd(m[(r * 4 + c) * 2], m[(r * 4 + c) * 2 + 1], x[c], acc);
          st[idx[r]] = acc;
        }
      }
      return;
    }
    default:
      return;
  }
}

// The reference's cumulative probabilities (measurement.c:281-283: a
// left-to-right FP64 sum of fl(cabs(a_i)^2), cabs = glibc hypot) by thread
// 0 in index order, then every shot by binary search: the first i with
// u < cum_i, else the last index with non-zero probability (0 if none) --
// measurement_all_qubits(u) bit for bit.  uni(k) is shot k's uniform,
// out(k, i) stores its outcome.  Ends with a barrier.
template <typename A, typename UniF, typename OutF>
__device__ void cdf_and_shots(const A* st, double* cum, unsigned int* last_nz, uint32_t n, uint32_t shots, UniF uni,
                              OutF out) {
  const uint32_t dim = 1u << n;
  if (threadIdx.x == 0) {
    double s = 0.0;
    unsigned int lnz = 0;
    bool any = false;
    for (uint32_t i = 0; i < dim; i++) {
      const double h = glibc_cabs((double)st[i].x, (double)st[i].y);
      const double p = __dmul_rn(h, h);
      if (p > 0.0) {
        lnz = i;
        any = true;
      }
      s = __dadd_rn(s, p);
      cum[i] = s;
    }
    *last_nz = any ? lnz : 0u;
  }
  __syncthreads();
  for (uint32_t sh = threadIdx.x; sh < shots; sh += blockDim.x) {
    const double u = uni(sh);
    uint32_t lo = 0, hi = dim;  // first i with u < cum[i]
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (u < cum[mid]) hi = mid;
      else lo = mid + 1;
    }
    out(sh, lo < dim ? lo : *last_nz);
  }
  __syncthreads();
}

}  // namespace small
}  // namespace mlb
