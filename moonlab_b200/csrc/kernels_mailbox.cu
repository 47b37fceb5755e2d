// kernels_mailbox.cu -- the persistent request loop for small circuits
// (<= 12 qubits complex128, <= 13 complex64): one launch serves requests as
// the host posts them, instead of one launch per gathered batch.
//
// Mailbox (device memory, written by the host's copy stream): a ring of
// request descriptors, a per-slot op region and uniform region, and the
// published count `tail`.  The host copies a request into its slot and then
// writes the new tail, both on one stream, so a block that reads tail with
// an acquire load sees the request's data in L2.  Every mailbox read goes
// to L2 (ld.global.cg, or the acquire load): a slot's addresses are
// rewritten by the copy engine while the kernel runs, and the SM's L1 is
// not kept coherent with those writes.
//
// Each block (256 threads, the state and its cumulative sums in shared
// memory) claims the next published request with a compare-and-swap on
// `head` (only below tail, so a claim is never left behind), runs it as
// kernels_small.cu does -- |0...0>, the ops staged through shared memory,
// the reference's sequential cumulative sum, every shot bit-identical to
// measurement_all_qubits(u) -- writes the outcomes into mapped host memory
// and then the slot's done word (the request's sequence number + 1) with a
// system-scope release, which the host polls.
//
// Waits are bounded: a block that finds no request for idle_ns of
// %globaltimer, or sees the stop word, exits; the last block out records
// whether the launch ended idle (MLB_ERR_TIMEOUT) or stopped.  The host
// relaunches the loop when it posts a request after the kernel has ended,
// so no block ever waits without limit.
#include <atomic>

#include "mlb_internal.h"
#include "small_circuit.cuh"

namespace mlb {

namespace {

using namespace small;

constexpr int kOpChunk = 32;  // ops staged into shared memory at a time

__device__ __forceinline__ uint64_t mb_ld_acquire(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t mb_ld_acquire32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void mb_st_release_sys(uint64_t* p, uint64_t v) {
  asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t mb_now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename Real>
__global__ void __launch_bounds__(kST) k_mailbox(MailboxDev mb) {
  using A = typename Cplx<Real>::T;
  extern __shared__ __align__(16) unsigned char sraw[];
  A* st = reinterpret_cast<A*>(sraw);
  double* cum = reinterpret_cast<double*>(sraw + sizeof(A) * (1u << mb.nmax));
  mlb_op_t* sops = reinterpret_cast<mlb_op_t*>(sraw + (sizeof(A) + sizeof(double)) * (1u << mb.nmax));
  __shared__ unsigned int last_nz;
  __shared__ uint64_t s_seq;
  __shared__ MailboxItem s_item;
  bool idle = false;
  for (;;) {
    if (threadIdx.x == 0) {
      // claim the next published request (bounded wait for one to arrive)
      uint64_t seq = ~0ull;
      const uint64_t t0 = mb_now_ns();
      for (;;) {
        const uint64_t tail = mb_ld_acquire(mb.tail);
        uint64_t h = mb_ld_acquire(mb.head);
        bool got = false;
        while (h < tail) {
          const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(mb.head),
                                                    (unsigned long long)h, (unsigned long long)(h + 1));
          if (prev == h) {
            got = true;
            break;
          }
          h = prev;
        }
        if (got) {
          seq = h;
          break;
        }
        if (mb_ld_acquire32(mb.stop)) break;
        if (mb_now_ns() - t0 > mb.idle_ns) {
          idle = true;
          break;
        }
        __nanosleep(2000);
      }
      s_seq = seq;
      if (seq != ~0ull) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(mb.items + seq % mb.slots);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s_item);
        for (int k = 0; k < (int)(sizeof(MailboxItem) / 4); k++) dst[k] = __ldcg(src + k);
      }
    }
    __syncthreads();
    const uint64_t seq = s_seq;
    if (seq == ~0ull) break;
    const MailboxItem item = s_item;
    const uint32_t slot = (uint32_t)(seq % mb.slots);
    const uint32_t dim = 1u << item.n;
    for (uint32_t i = threadIdx.x; i < dim; i += kST) st[i] = mk((Real)(i == 0 ? 1 : 0), (Real)0);
    const mlb_op_t* ops = mb.ops + (size_t)slot * mb.max_ops;
    for (uint32_t k0 = 0; k0 < item.num_ops; k0 += kOpChunk) {
      const uint32_t cnt = item.num_ops - k0 < (uint32_t)kOpChunk ? item.num_ops - k0 : (uint32_t)kOpChunk;
      // stage this chunk of ops through L2 (the slot is rewritten by copies)
      const uint64_t* src = reinterpret_cast<const uint64_t*>(ops + k0);
      uint64_t* dst = reinterpret_cast<uint64_t*>(sops);
      const uint32_t words = cnt * (uint32_t)(sizeof(mlb_op_t) / 8);
      __syncthreads();  // the previous chunk (and the |0...0> fill) are done
      for (uint32_t w = threadIdx.x; w < words; w += kST) dst[w] = __ldcg(src + w);
      __syncthreads();
      for (uint32_t k = 0; k < cnt; k++) {
        apply_op(st, item.n, sops[k]);
        __syncthreads();
      }
    }
    __syncthreads();
    const double* uni = mb.uniforms + (size_t)slot * mb.max_shots;
    unsigned long long* out = mb.outcomes + (size_t)slot * mb.max_shots;
    cdf_and_shots(
        st, cum, &last_nz, item.n, item.shots, [&](uint32_t k) { return __ldcg(uni + k); },
        [&](uint32_t k, unsigned int v) { out[k] = v; });
    // every thread's outcome writes before the done word (system scope: the
    // host reads both)
    __threadfence_system();
    __syncthreads();
    if (threadIdx.x == 0) mb_st_release_sys(mb.done + slot, seq + 1);
  }
  // the last block out records how the launch ended
  if (threadIdx.x == 0) {
    const unsigned int left = atomicAdd(mb.exited, 1u) + 1u;
    if (left == gridDim.x) *mb.end_status = idle ? MLB_ERR_TIMEOUT : MLB_OK;
  }
}

}  // namespace

static_assert(sizeof(mlb_op_t) % 8 == 0, "ops are staged as 8-byte words");
static_assert(sizeof(MailboxItem) % 4 == 0, "descriptors are read as 4-byte words");

size_t mailbox_smem_bytes(int dtype) {
  const uint32_t nmax = (uint32_t)small_max_qubits(dtype);
  const size_t amp = dtype == MLB_C128 ? 16 : 8;
  return (amp + sizeof(double)) * ((size_t)1 << nmax) + kOpChunk * sizeof(mlb_op_t);
}

int launch_mailbox(int dtype, const MailboxDev& mb, int ctas, cudaStream_t stream) {
  if (ctas < 1 || mb.slots < 1 || mb.nmax != (uint32_t)small_max_qubits(dtype)) return MLB_ERR_INVALID_ARG;
  const size_t smem = mailbox_smem_bytes(dtype);
  static std::atomic<uint64_t> attr_set_mask{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set_mask.load(std::memory_order_acquire) & bit)) {
    cudaFuncSetAttribute(k_mailbox<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mailbox_smem_bytes(MLB_C128));
    cudaFuncSetAttribute(k_mailbox<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)mailbox_smem_bytes(MLB_C64));
    attr_set_mask.fetch_or(bit, std::memory_order_release);
  }
  if (dtype == MLB_C128) k_mailbox<double><<<ctas, kST, smem, stream>>>(mb);
  else k_mailbox<float><<<ctas, kST, smem, stream>>>(mb);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb
