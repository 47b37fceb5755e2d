// kernels_fused.cu -- the fused complex64 path: dense 5-qubit blocks applied
// on the 5th-generation tensor cores (tcgen05) with split-bf16 products and
// FP32 accumulation in tensor memory.
//
// One pass streams the state once through shared memory in tiles of 2^13
// amplitudes (qubits 0..4 plus 8 chosen high qubits).  For a block acting on
// tile bits P (5 of them) the tile is a 256 x 32 complex matrix T[m][r]
// (m over the other 8 tile bits, r over P) and the block computes
// T <- T U^T.  In real arithmetic with A = [Re T | Im T] (256 x 64) and
// U' = [Re U  -Im U; Im U  Re U] (64 x 64):  [Re T' | Im T'] = A U'^T.
// Split precision: A = Ah + Al and U' = Uh + Ul with bf16 parts, and
//   A U'^T ~ Ah Uh^T + Al Uh^T + Ah Ul^T
// (the dropped Al Ul^T term is ~2^-16 of the result), accumulated in FP32.
// Each product is one K = 64 chunk, so a block is, per 128-row half,
// 3 x 4 tcgen05.mma of M = 128, N = 64, K = 16, issued by one thread into a
// 128-lane x 64-column FP32 accumulator in tensor memory.
//
// Per block: every thread (one per tile row m) converts its 32 amplitudes
// from the FP32 tile into the bf16 operand rows (K-major, 128-byte swizzle),
// the block's operand image (prepared on the host, 16 KiB) is copied in, one
// thread issues the MMAs and commits them to an mbarrier, and after the
// commit arrives every warp reads its 32 accumulator lanes back
// (tcgen05.ld 32x32b, 64 columns) into the FP32 tile.
//
// The completion wait is bounded: if it runs out the kernel sets *err,
// waits once more (bounded) for the MMAs in flight, frees its tensor memory
// and returns.
#include <atomic>

#include <cuda_bf16.h>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

constexpr int kFThreads = 256;
constexpr int kTileAmps = 1 << 13;
// shared-memory layout (bytes from a 1024-byte aligned base)
constexpr uint32_t kAHi = 0;          // 256 rows x 128 B
constexpr uint32_t kALo = 32768;
constexpr uint32_t kBHi = 65536;      // 64 rows x 128 B
constexpr uint32_t kBLo = 73728;
constexpr uint32_t kTile = 81920;     // 2^13 float2 = 64 KiB
constexpr uint32_t kMbar = 147456;
constexpr uint32_t kTmemSlot = 147464;
constexpr uint32_t kFlag = 147468;
constexpr uint32_t kSmemUsed = 147472;
constexpr uint32_t kSmemBytes = kSmemUsed + 1024;  // alignment slack
constexpr uint32_t kTmemCols = 128;
constexpr long long kWaitLimit = 1ll << 22;      // try_wait rounds before giving up

// instruction descriptor: D = F32, A = B = BF16, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B
// apart (SBO), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;               // leading byte offset (unused for this layout)
  d |= (uint64_t)(1024u >> 4) << 32;    // stride byte offset
  d |= (uint64_t)1 << 46;               // descriptor version
  d |= (uint64_t)2 << 61;               // SWIZZLE_128B
  return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; i++)
    if (mbar_try(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
  uint32_t* r = reinterpret_cast<uint32_t*>(v);
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,"
      "%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
      "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]),
        "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]),
        "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]),
        "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]),
        "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// XOR swizzle of the FP32 tile: spreads rows of any stride over the banks.
__device__ __forceinline__ uint32_t tsw(uint32_t e) { return e ^ (((e >> 5) ^ (e >> 10)) & 31u); }

__device__ __forceinline__ uint32_t deposit8(uint32_t v, const uint8_t (&pos)[8]) {
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) r |= ((v >> i) & 1u) << pos[i];
  return r;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

__global__ void __launch_bounds__(kFThreads, 1)
    k_fused(float2* __restrict__ amp, FusedPassDev pass, const FusedBlockDev* __restrict__ blocks,
            const uint8_t* __restrict__ images, int* __restrict__ err) {
  extern __shared__ uint8_t smraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(sm);
  float2* tile = reinterpret_cast<float2*>(sm + kTile);
  volatile int* flag = reinterpret_cast<volatile int*>(sm + kFlag);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar = sbase + kMbar;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + kTmemSlot),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *flag = 0;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kTmemSlot);

  // high tile bits -> global qubits; the remaining qubits enumerate tiles
  uint64_t hmask = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) hmask |= 1ull << pass.hbits[i];
  const uint64_t tmask = ~(hmask | 31ull);

  uint32_t phase = 0;
  bool bad = false;
  for (uint64_t t = blockIdx.x; t < pass.num_tiles && !bad; t += gridDim.x) {
    // global base of tile t: deposit t over the qubits outside the tile
    uint64_t gbase = 0;
    {
      uint64_t v = t, m = tmask;
      while (v && m) {
        const uint64_t low = m & (~m + 1);
        if (v & 1ull) gbase |= low;
        v >>= 1;
        m &= m - 1;
      }
    }
    // load: pairs of amplitudes (16 B), 32 contiguous per high combination
#pragma unroll 4
    for (int i = 0; i < kTileAmps / 2 / kFThreads; i++) {
      const uint32_t e = (uint32_t)(i * kFThreads + tid) * 2u;
      uint64_t g = gbase | (e & 31u);
#pragma unroll
      for (int h = 0; h < 8; h++) g |= (uint64_t)((e >> (5 + h)) & 1u) << pass.hbits[h];
      const float4 v = __ldcs(reinterpret_cast<const float4*>(amp + g));
      tile[tsw(e)] = make_float2(v.x, v.y);
      tile[tsw(e + 1)] = make_float2(v.z, v.w);
    }
    __syncthreads();

    for (uint32_t b = 0; b < pass.num_blocks && !bad; b++) {
      const FusedBlockDev blk = blocks[pass.block_begin + b];
      // operand image of U' (hi, lo) -> shared memory, 16 KiB
      {
        const uint4* src = reinterpret_cast<const uint4*>(images + (size_t)blk.image * 16384);
        uint4* dst = reinterpret_cast<uint4*>(sm + kBHi);
#pragma unroll
        for (int i = 0; i < 16384 / 16 / kFThreads; i++) dst[i * kFThreads + tid] = __ldg(src + i * kFThreads + tid);
      }
      // amplitude operand: this thread's row m = tid
      {
        const uint32_t m = (uint32_t)tid;
        const uint32_t ebase = deposit8(m, blk.q);
        uint32_t roff[32];
#pragma unroll
        for (int r = 0; r < 32; r++) {
          uint32_t o = 0;
#pragma unroll
          for (int j = 0; j < 5; j++) o |= (uint32_t)((r >> j) & 1) << blk.pos[j];
          roff[r] = o;
        }
        uint8_t* ahi = sm + kAHi + m * 128;
        uint8_t* alo = sm + kALo + m * 128;
        const uint32_t sx = m & 7u;
#pragma unroll
        for (int c = 0; c < 4; c++) {  // chunk c: r = 8c .. 8c+7
          uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
          for (int w = 0; w < 4; w++) {
            const float2 a0 = tile[tsw(ebase | roff[8 * c + 2 * w])];
            const float2 a1 = tile[tsw(ebase | roff[8 * c + 2 * w + 1])];
            const __nv_bfloat162 hre = __floats2bfloat162_rn(a0.x, a1.x);
            const __nv_bfloat162 him = __floats2bfloat162_rn(a0.y, a1.y);
            const float2 fre = __bfloat1622float2(hre), fim = __bfloat1622float2(him);
            rh[w] = *reinterpret_cast<const uint32_t*>(&hre);
            ih[w] = *reinterpret_cast<const uint32_t*>(&him);
            rl[w] = pack_bf16x2(a0.x - fre.x, a1.x - fre.y);
            il[w] = pack_bf16x2(a0.y - fim.x, a1.y - fim.y);
          }
          *reinterpret_cast<uint4*>(ahi + (((uint32_t)c ^ sx) << 4)) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
          *reinterpret_cast<uint4*>(ahi + (((uint32_t)(c + 4) ^ sx) << 4)) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
          *reinterpret_cast<uint4*>(alo + (((uint32_t)c ^ sx) << 4)) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
          *reinterpret_cast<uint4*>(alo + (((uint32_t)(c + 4) ^ sx) << 4)) = make_uint4(il[0], il[1], il[2], il[3]);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();

      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
        for (int h = 0; h < 2; h++) {
#pragma unroll
          for (int kc = 0; kc < 3; kc++) {
            const uint32_t a0 = sbase + (kc == 1 ? kALo : kAHi) + (uint32_t)h * 16384u;
            const uint32_t b0 = sbase + (kc == 2 ? kBLo : kBHi);
#pragma unroll
            for (int kk = 0; kk < 4; kk++)
              mma_bf16(tmem + (uint32_t)h * 64u, sdesc(a0 + kk * 32), sdesc(b0 + kk * 32),
                       (kc | kk) != 0 ? 1u : 0u);
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                     : "memory");
        if (!mbar_wait_bounded(bar, phase)) *flag = 1;
      }
      __syncthreads();
      if (*flag) {
        bad = true;
        break;
      }
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      {
        const uint32_t h = (uint32_t)warp >> 2, qd = (uint32_t)warp & 3u;
        float d[64];
        tmem_ld64(tmem + ((qd * 32u) << 16) + h * 64u, d);
        const uint32_t m = h * 128u + qd * 32u + (uint32_t)lane;
        const uint32_t ebase = deposit8(m, blk.q);
#pragma unroll
        for (int r = 0; r < 32; r++) {
          uint32_t o = 0;
#pragma unroll
          for (int j = 0; j < 5; j++) o |= (uint32_t)((r >> j) & 1) << blk.pos[j];
          tile[tsw(ebase | o)] = make_float2(d[r], d[32 + r]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncthreads();
    }
    if (bad) break;

    // store
#pragma unroll 4
    for (int i = 0; i < kTileAmps / 2 / kFThreads; i++) {
      const uint32_t e = (uint32_t)(i * kFThreads + tid) * 2u;
      uint64_t g = gbase | (e & 31u);
#pragma unroll
      for (int h = 0; h < 8; h++) g |= (uint64_t)((e >> (5 + h)) & 1u) << pass.hbits[h];
      const float2 a = tile[tsw(e)], c = tile[tsw(e + 1)];
      __stcs(reinterpret_cast<float4*>(amp + g), make_float4(a.x, a.y, c.x, c.y));
    }
    __syncthreads();
  }

  if (bad) {
    if (tid == 0) {
      atomicExch(err, 1);
      mbar_wait_bounded(bar, phase);  // let MMAs in flight finish before freeing
    }
    __syncthreads();
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

int launch_fused_pass(void* amp, int n, const FusedPassDev& pass, const FusedBlockDev* d_blocks,
                      const uint8_t* d_images, int* d_err, int num_sms, cudaStream_t stream) {
  if (n < 13 || pass.num_blocks == 0) return MLB_ERR_INVALID_ARG;
  static std::atomic<uint64_t> attr_set_mask{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set_mask.load(std::memory_order_acquire) & bit)) {
    cudaFuncSetAttribute(k_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    attr_set_mask.fetch_or(bit, std::memory_order_release);
  }
  uint64_t grid = (uint64_t)num_sms;
  if (grid > pass.num_tiles) grid = pass.num_tiles;
  k_fused<<<(unsigned)grid, kFThreads, kSmemBytes, stream>>>(reinterpret_cast<float2*>(amp), pass, d_blocks,
                                                             d_images, d_err);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb
