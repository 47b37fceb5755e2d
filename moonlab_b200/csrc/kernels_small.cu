// kernels_small.cu -- many small circuits in one launch (the serving path's
// small size classes: <= 12 qubits complex128, <= 13 qubits complex64).
//
// A small state fits one CTA's shared memory, so a CTA runs a whole request:
// |0...0>, every op of its circuit (all threads, one op at a time), the
// cumulative probabilities and all its shots.  The cumulative sum is the
// reference's left-to-right FP64 sum of fl(cabs(a_i)^2) (measurement.c:
// 281-283, cabs = glibc hypot), computed by one thread in index order, so
// every shot is bit-identical to measurement_all_qubits(u): the first i with
// u < cum_i, else the last index with non-zero probability (0 if none).
// The launch is persistent over its items: CTA b takes items b, b + grid, ...
#include <atomic>

#include "kernels_common.cuh"
#include "hypot_glibc.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

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

template <typename Real>
__global__ void __launch_bounds__(kST) k_small(const SmallItem* __restrict__ items, int num_items,
                                               const mlb_op_t* __restrict__ ops,
                                               const double* __restrict__ uniforms,
                                               unsigned long long* __restrict__ outcomes, uint32_t nmax) {
  using A = typename Cplx<Real>::T;
  extern __shared__ __align__(16) unsigned char sraw[];
  A* st = reinterpret_cast<A*>(sraw);
  double* cum = reinterpret_cast<double*>(sraw + sizeof(A) * (1u << nmax));
  __shared__ unsigned int last_nz;
  for (int it = blockIdx.x; it < num_items; it += gridDim.x) {
    const SmallItem item = items[it];
    const uint32_t dim = 1u << item.n;
    for (uint32_t i = threadIdx.x; i < dim; i += kST) st[i] = mk((Real)(i == 0 ? 1 : 0), (Real)0);
    __syncthreads();
    for (uint32_t k = 0; k < item.num_ops; k++) {
      apply_op(st, item.n, ops[item.ops_off + k]);  // fields read from global memory (cached)
      __syncthreads();
    }
    if (threadIdx.x == 0) {  // the reference's sequential sum, in index order
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
      last_nz = any ? lnz : 0u;
    }
    __syncthreads();
    for (uint32_t sh = threadIdx.x; sh < item.shots; sh += kST) {
      const double u = uniforms[item.uni_off + sh];
      uint32_t lo = 0, hi = dim;  // first i with u < cum[i]
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (u < cum[mid]) hi = mid;
        else lo = mid + 1;
      }
      outcomes[item.out_off + sh] = lo < dim ? lo : last_nz;
    }
    __syncthreads();
  }
}

template <typename Real>
int launch_small_t(const SmallItem* d_items, int num_items, const mlb_op_t* d_ops, const double* d_uni,
                   unsigned long long* d_out, uint32_t nmax, int num_sms, cudaStream_t stream) {
  using A = typename Cplx<Real>::T;
  const size_t smem = (sizeof(A) + sizeof(double)) << nmax;
  static std::atomic<uint64_t> attr_set_mask{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set_mask.load(std::memory_order_acquire) & bit)) {
    const size_t max_smem = (sizeof(A) + sizeof(double)) << small_max_qubits(sizeof(A) == 16 ? MLB_C128 : MLB_C64);
    cudaFuncSetAttribute(k_small<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    attr_set_mask.fetch_or(bit, std::memory_order_release);
  }
  int grid = num_items < num_sms * 2 ? num_items : num_sms * 2;
  if (grid < 1) grid = 1;
  k_small<Real><<<grid, kST, smem, stream>>>(d_items, num_items, d_ops, d_uni, d_out, nmax);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace

int small_max_qubits(int dtype) { return dtype == MLB_C128 ? 12 : 13; }

int launch_small_circuits(int dtype, const SmallItem* d_items, int num_items, const mlb_op_t* d_ops,
                          const double* d_uniforms, unsigned long long* d_outcomes, uint32_t nmax, int num_sms,
                          cudaStream_t stream) {
  if (num_items < 1 || nmax < 1 || (int)nmax > small_max_qubits(dtype)) return MLB_ERR_INVALID_ARG;
  if (dtype == MLB_C128)
    return launch_small_t<double>(d_items, num_items, d_ops, d_uniforms, d_outcomes, nmax, num_sms, stream);
  return launch_small_t<float>(d_items, num_items, d_ops, d_uniforms, d_outcomes, nmax, num_sms, stream);
}

}  // namespace mlb
