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
#include "small_circuit.cuh"

namespace mlb {

namespace {

using namespace small;

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
    cdf_and_shots(
        st, cum, &last_nz, item.n, item.shots, [&](uint32_t k) { return uniforms[item.uni_off + k]; },
        [&](uint32_t k, unsigned int v) { outcomes[item.out_off + k] = v; });
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
