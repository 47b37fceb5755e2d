// kernels_reduce.cu -- FP64 reductions in one HBM pass.
//
// probs_z: the norm and P(qubit=1) for every qubit from a single read of the
// state (the reference makes one full pass per qubit, measurement.c:73).
// A CTA walks chunks of 2^13 contiguous amplitudes; in a chunk thread t
// reads amplitudes t + 256 k (k < 32), so the low 8 index bits are the
// thread's own (constant), bits 8..12 are the loop counter (compile-time
// after unrolling) and bits >= 13 are the chunk index (constant per chunk).
// Per amplitude that costs one |a|^2 and ~2.5 FP64 adds; the chunk totals go
// to a small buffer that a second kernel folds into the high-bit sums.
// All reductions use a fixed order, so results are identical run to run.
#include <algorithm>
#include <atomic>
#include <mutex>

#include "kernels_common.cuh"
#include "hypot_glibc.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

constexpr int kRT = 256;        // threads per CTA
constexpr int kRK = 32;         // amplitudes per thread per chunk
constexpr int kChunkBits = 13;  // 2^13 amplitudes per chunk

template <typename A> __device__ __forceinline__ double norm2(const A& a) {
  const double x = (double)a.x, y = (double)a.y;
  return x * x + y * y;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r += red[i];
  return r;  // valid in thread 0
}

// Pass 1: per-CTA sums for bits 0..12 (+ total) and per-chunk totals.
template <typename Real>
__global__ void __launch_bounds__(kRT) k_probs_z_pass1(const typename Cplx<Real>::T* __restrict__ amp,
                                                       uint64_t num_chunks, uint32_t chunk_amps,
                                                       double* __restrict__ chunk_tot,
                                                       double* __restrict__ partials) {
  __shared__ double red[kRT / 32];
  double low_tot = 0.0;                 // this thread's total (its low bits are fixed)
  double mid[kChunkBits - 8] = {0, 0, 0, 0, 0};
  for (uint64_t c = blockIdx.x; c < num_chunks; c += gridDim.x) {
    const uint64_t base = c << kChunkBits;
    double ctot = 0.0;
    if (chunk_amps == (1u << kChunkBits)) {
      double p[kRK];
#pragma unroll
      for (int k = 0; k < kRK; k++) p[k] = norm2(amp[base + threadIdx.x + (uint32_t)k * kRT]);
#pragma unroll
      for (int k = 0; k < kRK; k++) {
        ctot += p[k];
#pragma unroll
        for (int b = 0; b < kChunkBits - 8; b++)
          if (k >> b & 1) mid[b] += p[k];
      }
    } else {  // small state: a single partial chunk
      for (uint32_t e = threadIdx.x; e < chunk_amps; e += kRT) {
        const double p = norm2(amp[e]);
        ctot += p;
        const uint32_t k = e / kRT;
#pragma unroll
        for (int b = 0; b < kChunkBits - 8; b++)
          if (k >> b & 1) mid[b] += p;
      }
    }
    low_tot += ctot;
    const double t = block_sum(ctot, red);
    if (threadIdx.x == 0) chunk_tot[c] = t;
  }
  // Per-CTA partials: [0] total, [1+b] bit b for b < 13.
  double* out = partials + (size_t)blockIdx.x * (1 + kChunkBits);
  double v = block_sum(low_tot, red);
  if (threadIdx.x == 0) out[0] = v;
  for (int b = 0; b < 8; b++) {
    v = block_sum((threadIdx.x >> b & 1) ? low_tot : 0.0, red);
    if (threadIdx.x == 0) out[1 + b] = v;
  }
  for (int b = 0; b < kChunkBits - 8; b++) {
    v = block_sum(mid[b], red);
    if (threadIdx.x == 0) out[1 + 8 + b] = v;
  }
}

// Pass 2 (one CTA): fold CTA partials and chunk totals into out[0..n) = P1,
// out[n] = norm.
__global__ void __launch_bounds__(kRT) k_probs_z_pass2(const double* __restrict__ chunk_tot,
                                                       uint64_t num_chunks,
                                                       const double* __restrict__ partials,
                                                       int num_parts, int n,
                                                       double* __restrict__ out) {
  __shared__ double red[kRT / 32];
  // low bits and total from the CTA partials (fixed order)
  for (int j = 0; j < 1 + kChunkBits; j++) {
    double v = 0.0;
    for (int i = threadIdx.x; i < num_parts; i += kRT) v += partials[(size_t)i * (1 + kChunkBits) + j];
    v = block_sum(v, red);
    if (threadIdx.x == 0) {
      if (j == 0) out[n] = v;
      else if (j - 1 < n) out[j - 1] = v;
    }
  }
  // high bits from the chunk totals
  for (int b = kChunkBits; b < n; b++) {
    const int cb = b - kChunkBits;
    double v = 0.0;
    for (uint64_t c = threadIdx.x; c < num_chunks; c += kRT)
      if (c >> cb & 1ull) v += chunk_tot[c];
    v = block_sum(v, red);
    if (threadIdx.x == 0) out[b] = v;
  }
}

// <psi|P|psi> for Pauli strings sharing one X mask: P|i> = i^{ny}
// (-1)^{|i & z|} |i ^ x>.  Each pair (i, i^x) is read once; x = 0 gives the
// diagonal (Z-only) strings.  out[t] gets coeff_t * Re(...), summed later.
template <typename Real>
__global__ void __launch_bounds__(kRT) k_pauli(const typename Cplx<Real>::T* __restrict__ amp,
                                               int n, uint64_t xmask, int num_terms,
                                               const uint64_t* __restrict__ zmasks,
                                               const int* __restrict__ nys,
                                               double* __restrict__ partials) {
  __shared__ double red[kRT / 32];
  constexpr int kMaxT = 16;
  double acc[kMaxT];
#pragma unroll
  for (int t = 0; t < kMaxT; t++) acc[t] = 0.0;
  const uint64_t dim = 1ull << n;
  const int hb = xmask ? 63 - __clzll(xmask) : -1;
  const uint64_t items = xmask ? dim >> 1 : dim;
  const uint64_t stride = (uint64_t)gridDim.x * kRT;
  for (uint64_t j = (uint64_t)blockIdx.x * kRT + threadIdx.x; j < items; j += stride) {
    if (xmask) {
      const uint64_t lo = j & ((1ull << hb) - 1ull);
      const uint64_t i = ((j >> hb) << (hb + 1)) | lo;  // bit hb = 0
      const uint64_t k = i ^ xmask;
      const auto ai = amp[i], ak = amp[k];
      // conj(a_k) a_i and conj(a_i) a_k = conj of the former
      const double re = (double)ak.x * ai.x + (double)ak.y * ai.y;
      const double im = (double)ak.x * ai.y - (double)ak.y * ai.x;
#pragma unroll
      for (int t = 0; t < kMaxT; t++) {
        if (t >= num_terms) break;
        const uint64_t z = zmasks[t];
        const int ny = nys[t] & 3;
        const double si = parity64(i & z) ? -1.0 : 1.0;
        const double sk = parity64(k & z) ? -1.0 : 1.0;
        // term_i = i^ny si conj(a_k) a_i ; term_k = i^ny sk conj(a_i) a_k
        double tr_i, tr_k;
        switch (ny) {
          case 0: tr_i = re; tr_k = re; break;
          case 1: tr_i = -im; tr_k = im; break;
          case 2: tr_i = -re; tr_k = -re; break;
          default: tr_i = im; tr_k = -im; break;
        }
        acc[t] += si * tr_i + sk * tr_k;
      }
    } else {
      const auto a = amp[j];
      const double p = norm2(a);
#pragma unroll
      for (int t = 0; t < kMaxT; t++) {
        if (t >= num_terms) break;
        acc[t] += parity64(j & zmasks[t]) ? -p : p;
      }
    }
  }
  for (int t = 0; t < num_terms && t < kMaxT; t++) {
    const double v = block_sum(acc[t], red);
    if (threadIdx.x == 0) partials[(size_t)blockIdx.x * kMaxT + t] = v;
  }
}

__global__ void k_fold_partials(const double* __restrict__ partials, int num_parts, int stride,
                                int count, double* __restrict__ out) {
  __shared__ double red[kRT / 32];
  for (int j = 0; j < count; j++) {
    double v = 0.0;
    for (int i = threadIdx.x; i < num_parts; i += kRT) v += partials[(size_t)i * stride + j];
    v = block_sum(v, red);
    if (threadIdx.x == 0) out[j] = v;
  }
}

template <typename Real>
__global__ void k_probabilities(const typename Cplx<Real>::T* __restrict__ amp, uint64_t dim,
                                int rule, double* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
    const auto a = amp[i];
    const double x = (double)a.x, y = (double)a.y;
    if (rule == 0) {
      const double h = glibc_cabs(x, y);
      out[i] = __dmul_rn(h, h);
    } else {
      out[i] = __fma_rn(x, x, __dmul_rn(y, y));  // fma(re, re, im*im), as the reference build
    }
  }
}

// amp *= factor where (i & zero_mask) == zero_val, else amp = 0.
// zero_mask = 0 scales everything.  Division mode (factor < 0 encodes
// "divide by -factor") reproduces quantum_measure's amp /= norm.
template <typename Real>
__global__ void k_scale(typename Cplx<Real>::T* __restrict__ amp, uint64_t dim, double factor,
                        uint64_t keep_mask, uint64_t keep_val) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const bool divide = factor < 0.0;
  const double f = divide ? -factor : factor;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += stride) {
    auto a = amp[i];
    if ((i & keep_mask) != keep_val) {
      a.x = 0;
      a.y = 0;
    } else if (divide) {
      a.x = (Real)__ddiv_rn((double)a.x, f);
      a.y = (Real)__ddiv_rn((double)a.y, f);
    } else {
      a.x = (Real)__dmul_rn((double)a.x, f);
      a.y = (Real)__dmul_rn((double)a.y, f);
    }
    amp[i] = a;
  }
}

int rgrid(uint64_t items, int num_sms) {
  uint64_t g = (items + kRT - 1) / kRT;
  const uint64_t cap = (uint64_t)num_sms * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

int launch_reduce_probs_z(int dtype, const void* amp, int n, double* d_out, double* d_partials,
                          int num_sms, cudaStream_t stream) {
  const uint64_t dim = 1ull << n;
  const uint64_t num_chunks = n >= kChunkBits ? dim >> kChunkBits : 1;
  const uint32_t chunk_amps = n >= kChunkBits ? (1u << kChunkBits) : (uint32_t)dim;
  int grid = (int)std::min<uint64_t>(num_chunks, (uint64_t)num_sms * 4);
  // partials layout: [grid x 14] then chunk totals
  double* parts = d_partials;
  double* chunk_tot = d_partials + (size_t)grid * (1 + kChunkBits);
  if (dtype == MLB_C128)
    k_probs_z_pass1<double><<<grid, kRT, 0, stream>>>((const double2*)amp, num_chunks, chunk_amps,
                                                      chunk_tot, parts);
  else
    k_probs_z_pass1<float><<<grid, kRT, 0, stream>>>((const float2*)amp, num_chunks, chunk_amps,
                                                     chunk_tot, parts);
  k_probs_z_pass2<<<1, kRT, 0, stream>>>(chunk_tot, num_chunks, parts, grid, n, d_out);
  count_launch(2);
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

// Grouped Pauli expectation (called by the host with one X-mask group).
int launch_pauli_group(int dtype, const void* amp, int n, uint64_t xmask, int num_terms,
                       const uint64_t* d_zmasks, const int* d_nys, double* d_out_terms,
                       double* d_partials, int num_sms, cudaStream_t stream) {
  const uint64_t items = xmask ? (1ull << n) >> 1 : (1ull << n);
  const int grid = rgrid(items, num_sms);
  if (dtype == MLB_C128)
    k_pauli<double><<<grid, kRT, 0, stream>>>((const double2*)amp, n, xmask, num_terms, d_zmasks,
                                              d_nys, d_partials);
  else
    k_pauli<float><<<grid, kRT, 0, stream>>>((const float2*)amp, n, xmask, num_terms, d_zmasks,
                                             d_nys, d_partials);
  k_fold_partials<<<1, kRT, 0, stream>>>(d_partials, grid, 16, num_terms, d_out_terms);
  count_launch(2);
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

int launch_probabilities(int dtype, const void* amp, int n, int rule, double* d_out,
                         cudaStream_t stream) {
  const uint64_t dim = 1ull << n;
  const int grid = rgrid(dim, 148 * 4);
  if (dtype == MLB_C128)
    k_probabilities<double><<<grid, kRT, 0, stream>>>((const double2*)amp, dim, rule, d_out);
  else
    k_probabilities<float><<<grid, kRT, 0, stream>>>((const float2*)amp, dim, rule, d_out);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

int launch_scale(int dtype, void* amp, int n, double factor, uint64_t keep_mask, uint64_t keep_val,
                 cudaStream_t stream) {
  const uint64_t dim = 1ull << n;
  const int grid = rgrid(dim, 148 * 4);
  if (dtype == MLB_C128)
    k_scale<double><<<grid, kRT, 0, stream>>>((double2*)amp, dim, factor, keep_mask, keep_val);
  else
    k_scale<float><<<grid, kRT, 0, stream>>>((float2*)amp, dim, factor, keep_mask, keep_val);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb

// ---- probs_z without device allocation -------------------------------------
// mlb_prob_one_all_noalloc runs the probs_z reduction above on caller-owned
// buffers, with its scratch in one fixed array per device instead of a
// cudaMalloc'd buffer.  Scratch use: pass-1 partials ([grid x 14] doubles,
// grid <= kNoAllocMaxParts) followed by one total per 2^13-amplitude chunk
// (2^(n-13) doubles, at most 2^17 for n = 30).  Pass 1 writes every entry
// pass 2 reads, so nothing is cleared between calls.
namespace {

constexpr uint32_t kNoAllocMaxQubits = 30;
constexpr int kNoAllocMaxParts = 1024;  // pass-1 CTAs; the grid is min(chunks, 4 * SMs)
constexpr size_t kNoAllocScratchDoubles =
    (size_t)kNoAllocMaxParts * (1 + 13) + (size_t(1) << (kNoAllocMaxQubits - 13));  // 145,408
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_probs_z_scratch[kNoAllocScratchDoubles];

struct NoAllocDevice {
  std::atomic<double*> scratch{nullptr};
  int num_sms = 0;
};
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

// Set-up, once per device, with that device current: the array's address and
// the SM count.
int noalloc_setup(int dev, double** scratch, int* num_sms) {
  NoAllocDevice& d = g_noalloc_dev[dev];
  double* p = d.scratch.load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    p = d.scratch.load(std::memory_order_relaxed);
    if (!p) {
      int sms = 0;
      cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess || sms <= 0)
        return mlb::record_error(MLB_ERR_DRIVER, "mlb_prob_one_all_noalloc: SM count query failed");
      void* addr = nullptr;
      e = cudaGetSymbolAddress(&addr, g_probs_z_scratch);
      if (e != cudaSuccess || !addr)
        return mlb::record_error(MLB_ERR_DRIVER, "mlb_prob_one_all_noalloc: scratch address lookup failed");
      d.num_sms = sms;
      p = (double*)addr;
      d.scratch.store(p, std::memory_order_release);
    }
  }
  *scratch = p;
  *num_sms = d.num_sms;
  return MLB_OK;
}

// True when ptr is device (or managed) memory of device dev.
bool on_device(const void* ptr, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace

extern "C" int mlb_prob_one_all_noalloc(const void* amp_device, int dtype, uint32_t num_qubits,
                                        double* out_device, void* stream) {
  if (!amp_device || !out_device)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "mlb_prob_one_all_noalloc: null buffer");
  if (dtype != MLB_C128 && dtype != MLB_C64)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "mlb_prob_one_all_noalloc: dtype must be MLB_C128 or MLB_C64");
  if (num_qubits < 1 || num_qubits > kNoAllocMaxQubits)
    return mlb::record_error(MLB_ERR_NUM_QUBITS,
                             "mlb_prob_one_all_noalloc: num_qubits must be 1..30 (fixed scratch size)");
  const uintptr_t align = dtype == MLB_C128 ? 16 : 8;
  if ((uintptr_t)amp_device % align || (uintptr_t)out_device % 8)
    return mlb::record_error(MLB_ERR_INVALID_ARG, "mlb_prob_one_all_noalloc: misaligned buffer");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return mlb::record_error(MLB_ERR_NO_DEVICE, "mlb_prob_one_all_noalloc: no current device");
  }
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return mlb::record_error(MLB_ERR_NOT_SUPPORTED, "mlb_prob_one_all_noalloc: device ordinal above 63");
  if (!on_device(amp_device, dev) || !on_device(out_device, dev))
    return mlb::record_error(MLB_ERR_INVALID_ARG,
                             "mlb_prob_one_all_noalloc: buffers must be device memory of the current device");
  double* scratch = nullptr;
  int num_sms = 0;
  int rc = noalloc_setup(dev, &scratch, &num_sms);
  if (rc) return rc;
  // grid = min(chunks, 4 * SMs) stays within the array's kNoAllocMaxParts CTAs.
  const int sms = std::min(num_sms, kNoAllocMaxParts / 4);
  rc = mlb::launch_reduce_probs_z(dtype, amp_device, (int)num_qubits, out_device, scratch, sms,
                                  (cudaStream_t)stream);
  if (rc) return mlb::record_error(rc, "mlb_prob_one_all_noalloc: launch failed");
  return MLB_OK;
}
