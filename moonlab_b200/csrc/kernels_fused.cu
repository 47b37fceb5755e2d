// kernels_fused.cu -- the fused complex64 path: dense 5-qubit blocks applied
// on the 5th-generation tensor cores (tcgen05) with split-bf16 products and
// FP32 accumulation in tensor memory.
//
// One pass streams the state once through shared memory in tiles of 2^13
// amplitudes (the low qubits, contiguous in memory, plus chosen high qubits).  For a block acting on
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
// from the FP32 tile into its row of the bf16 amplitude operand and stores
// it to tensor memory (tcgen05.st, row per lane, two bf16 per column: the
// operand-A layout of an A-from-TMEM MMA); the block's U' image (prepared
// on the host, 16 KiB, K-major 128-byte swizzle) comes into shared memory;
// one thread issues the MMAs and commits them to an mbarrier, and after the
// commit arrives every warp reads its 32 accumulator lanes back
// (tcgen05.ld 32x32b, 64 columns) into the FP32 tile.
//
// Occupancy: a CTA of 4 warps (each warp owns one tensor-memory lane quadrant
// and handles one row of each 128-row half) holds one tile buffer, the
// block's operand image and 256 TMEM columns, so two CTAs share an SM: one
// CTA's MMA waits and tile loads (16-byte async copies, cp.async) overlap
// the other's operand conversion and readback.  Each block's operand image
// comes by one bulk copy completing on its own mbarrier, requested as soon
// as the previous block's MMAs have completed.
//
// Waits are bounded: if one runs out the kernel sets *err, waits once more
// (bounded) for what it issued, frees its tensor memory and returns.
#include <atomic>

#include <cuda_bf16.h>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

constexpr int kFThreads = 128;       // 4 warps: each owns one TMEM lane quadrant (both halves)
constexpr int kTileAmps = 1 << 13;
constexpr int kPairsPerThread = kTileAmps / 2 / kFThreads;  // 32
// shared-memory layout (bytes from a 1024-byte aligned base); two CTAs per SM
constexpr uint32_t kBHi = 0;          // 64 rows x 128 B, then lo
constexpr uint32_t kBLo = 8192;
constexpr uint32_t kTile0 = 16384;    // one tile buffer of 2^13 float2 (64 KiB)
constexpr uint32_t kTileBytes = 65536;
constexpr uint32_t kMbarMma = 81920;  // two: one per 128-row half
constexpr uint32_t kMbarB = 81936;
constexpr uint32_t kTmemSlot = 81944;
constexpr uint32_t kFlag = 81948;
constexpr uint32_t kRoff = 81952;     // per block: 32 swizzled column offsets (uint16), 16-byte aligned
constexpr int kMaxBlocks = 64;        // blocks per pass (the planner splits longer passes)
constexpr uint32_t kHiDep = kRoff + kMaxBlocks * 64;  // 32 x uint64: global offsets of tile bits 8..12
constexpr uint32_t kSmemUsed = kHiDep + kPairsPerThread * 8;
constexpr uint32_t kSmemBytes = kSmemUsed + 1024;  // alignment slack
constexpr uint32_t kTmemCols = 256;  // D: columns 0..127 (64 per half); A: 128..255
constexpr uint32_t kACol = 128;      // A of half h: hi at kACol + 64 h, lo at kACol + 64 h + 32
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

// A from tensor memory (row per lane, K packed two bf16 per column), B from
// shared memory.
__device__ __forceinline__ void mma_bf16_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// 32 consecutive columns of this thread's lane.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
      "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]),
      "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]),
      "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
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

// 16 KiB operand image (global, L2-resident) -> shared memory by one bulk
// copy that completes on mbarrier `bar` (one thread).
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "{\n\t"
      ".reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 st, [%0], %1;\n\t"
      "}\n" ::"r"(bar),
      "r"(bytes)
      : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
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

// XOR swizzle of the FP32 tile on bits 1..4 (pairs of amplitudes stay
// together, so 16-byte async copies land whole): spreads rows of any stride
// over the banks.
__device__ __forceinline__ uint32_t tsw(uint32_t e) { return e ^ ((((e >> 5) ^ (e >> 9)) & 15u) << 1); }

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

__device__ __forceinline__ uint64_t tile_base(uint64_t t, uint64_t tmask) {
  uint64_t gbase = 0, v = t, m = tmask;
  while (v && m) {
    const uint64_t low = m & (~m + 1);
    if (v & 1ull) gbase |= low;
    v >>= 1;
    m &= m - 1;
  }
  return gbase;
}

// Amplitude pair (e, e+1) of a tile -> its global index.
__device__ __forceinline__ uint64_t tile_global(uint64_t gbase, uint32_t e, const FusedPassDev& pass) {
  const uint32_t L = pass.num_low;
  uint64_t g = gbase | (e & ((1u << L) - 1u));
#pragma unroll
  for (int h = 0; h < 12; h++)
    if (h < (int)pass.num_high) g |= (uint64_t)((e >> (L + h)) & 1u) << pass.hbits[h];
  return g;
}

__global__ void __launch_bounds__(kFThreads, 2)
    k_fused(float2* __restrict__ amp, FusedPassDev pass, const FusedBlockDev* __restrict__ blocks,
            const uint8_t* __restrict__ images, int* __restrict__ err) {
  extern __shared__ uint8_t smraw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbase = smem_u32(sm);
  volatile int* flag = reinterpret_cast<volatile int*>(sm + kFlag);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar_mma = sbase + kMbarMma, bar_b = sbase + kMbarB;  // bar_mma + 8 h: half h

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + kTmemSlot),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_mma), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_mma + 8), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_b), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *flag = 0;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kTmemSlot);

  // Column offsets of every block of the pass, swizzled once: tsw is linear
  // over GF(2), so tsw(row | col) = tsw(row) ^ tsw(col) for disjoint bits.
  uint16_t* roff_tab = reinterpret_cast<uint16_t*>(sm + kRoff);
  for (uint32_t i = tid; i < pass.num_blocks * 32u; i += kFThreads) {
    const FusedBlockDev blk = blocks[pass.block_begin + i / 32u];
    const uint32_t r = i & 31u;
    uint32_t o = 0;
#pragma unroll
    for (int j = 0; j < 5; j++) o |= ((r >> j) & 1u) << blk.pos[j];
    roff_tab[i] = (uint16_t)tsw(o);
  }
  if (tid < kPairsPerThread)
    reinterpret_cast<uint64_t*>(sm + kHiDep)[tid] = tile_global(0, (uint32_t)tid * 2u * kFThreads, pass);
  __syncthreads();

  uint64_t hmask = (1ull << pass.num_low) - 1ull;
#pragma unroll
  for (int i = 0; i < 12; i++)
    if (i < (int)pass.num_high) hmask |= 1ull << pass.hbits[i];
  const uint64_t tmask = ~hmask;

  // Tile-local index e of this thread's i-th amplitude pair: e = 512 i + 2 tid.
  // Its global offset is linear in e over disjoint bits, so it splits into
  // a per-thread part (bits 0..8) and a per-i part (bits 9..12, shared table).
  const uint64_t my_off = tile_global(0, 2u * (uint32_t)tid, pass);
  const uint64_t* hidep = reinterpret_cast<const uint64_t*>(sm + kHiDep);
  // tsw is linear over GF(2): tsw(256 i + 2 tid) = tsw(256 i) ^ tsw(2 tid), the
  // first term a compile-time constant in the unrolled loops
  const uint32_t my_sw0 = tsw(2u * (uint32_t)tid);

  auto load_tile = [&](uint64_t t) {
    const uint64_t gb = tile_base(t, tmask) | my_off;
    const uint32_t dst0 = sbase + kTile0;
#pragma unroll 8
    for (int i = 0; i < kPairsPerThread; i++) cp_async16(dst0 + (my_sw0 ^ tsw((uint32_t)i * 2u * kFThreads)) * 8u, amp + (gb | hidep[i]));
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };

  uint32_t ph_mma = 0, ph_b = 0;
  bool bad = false;
  if (tid == 0 && (uint64_t)blockIdx.x < pass.num_tiles)
    bulk_load(sbase + kBHi, images + (size_t)blocks[pass.block_begin].image * 16384, 16384, bar_b);
  float2* tile = reinterpret_cast<float2*>(sm + kTile0);
  for (uint64_t t = blockIdx.x; t < pass.num_tiles && !bad; t += gridDim.x) {
    load_tile(t);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();

    for (uint32_t b = 0; b < pass.num_blocks; b++) {
      const FusedBlockDev blk = blocks[pass.block_begin + b];
      // amplitude operand: this thread's rows m = tid and 128 + tid
#pragma unroll 1
      for (uint32_t hh = 0; hh < 2; hh++) {
        const uint32_t m = 128u * hh + (uint32_t)tid;
        const uint32_t ebase = tsw(deposit8(m, blk.q));
        uint32_t roff[32];
        {
          const uint4* rt = reinterpret_cast<const uint4*>(roff_tab + b * 32u);
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const uint4 x = rt[v];
            const uint32_t w4[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
              roff[v * 8 + 2 * k] = w4[k] & 0xffffu;
              roff[v * 8 + 2 * k + 1] = w4[k] >> 16;
            }
          }
        }
        // row m's operand words: word j holds K elements 2j, 2j+1 (re of r for
        // K < 32, im of r - 32 above), hi and lo parts
        uint32_t whi[32], wlo[32];
#pragma unroll
        for (int c = 0; c < 4; c++) {
#pragma unroll
          for (int w = 0; w < 4; w++) {
            const float2 a0 = tile[ebase ^ roff[8 * c + 2 * w]];
            const float2 a1 = tile[ebase ^ roff[8 * c + 2 * w + 1]];
            const __nv_bfloat162 hre = __floats2bfloat162_rn(a0.x, a1.x);
            const __nv_bfloat162 him = __floats2bfloat162_rn(a0.y, a1.y);
            const float2 fre = __bfloat1622float2(hre), fim = __bfloat1622float2(him);
            whi[4 * c + w] = *reinterpret_cast<const uint32_t*>(&hre);
            whi[16 + 4 * c + w] = *reinterpret_cast<const uint32_t*>(&him);
            wlo[4 * c + w] = pack_bf16x2(a0.x - fre.x, a1.x - fre.y);
            wlo[16 + 4 * c + w] = pack_bf16x2(a0.y - fim.x, a1.y - fim.y);
          }
        }
        // this warp's lane quadrant: row m = 128 h + 32 qd + lane
        const uint32_t h = m >> 7, qd = (m >> 5) & 3u;
        const uint32_t ta = tmem + ((qd * 32u) << 16) + kACol + h * 64u;
        tmem_st32(ta, whi);
        tmem_st32(ta + 32u, wlo);
        asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncthreads();

      if (tid == 0) {
        if (mbar_wait_bounded(bar_b, ph_b)) {  // operand image landed
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
          for (int h = 0; h < 2; h++) {
#pragma unroll
            for (int kc = 0; kc < 3; kc++) {
              const uint32_t a0 = tmem + kACol + (uint32_t)h * 64u + (kc == 1 ? 32u : 0u);
              const uint32_t b0 = sbase + (kc == 2 ? kBLo : kBHi);
#pragma unroll
              for (int kk = 0; kk < 4; kk++)
                mma_bf16_ts(tmem + (uint32_t)h * 64u, a0 + kk * 8u, sdesc(b0 + kk * 32),
                            (kc | kk) != 0 ? 1u : 0u);
            }
            // half h done -> its mbarrier (commit covers all earlier MMAs of this thread)
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             bar_mma + 8u * (uint32_t)h)
                         : "memory");
          }
        } else {
          atomicOr((int*)flag, 1);  // operand copy not seen; no MMA issued
        }
      }
      // Each warp owns lane quadrant qd: half 0 first, then half 1 (half 0's
      // readback overlaps half 1's MMAs); the lane that sees half 1 complete
      // requests the next operand image.
      {
        const uint32_t qd = (uint32_t)warp;
        __syncwarp();
#pragma unroll 1
        for (uint32_t h = 0; h < 2; h++) {
          int ok = 0;
          if (lane == 0 && !*flag) {
            ok = mbar_wait_bounded(bar_mma + 8u * h, ph_mma) ? 1 : 0;
            if (!ok) atomicOr((int*)flag, 2);
            if (ok && h == 1 && qd == 0) {
              const bool more = b + 1 < pass.num_blocks || t + gridDim.x < pass.num_tiles;
              const uint32_t nb = b + 1 < pass.num_blocks ? b + 1 : 0;
              if (more)
                bulk_load(sbase + kBHi, images + (size_t)blocks[pass.block_begin + nb].image * 16384, 16384,
                          bar_b);
            }
          }
          ok = __shfl_sync(0xffffffffu, ok, 0);
          if (!ok) break;
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          float d[64];
          tmem_ld64(tmem + ((qd * 32u) << 16) + h * 64u, d);
          const uint32_t m = h * 128u + qd * 32u + (uint32_t)lane;
          const uint32_t ebase = tsw(deposit8(m, blk.q));
          const uint4* rt = reinterpret_cast<const uint4*>(roff_tab + b * 32u);
#pragma unroll
          for (int v = 0; v < 4; v++) {
            const uint4 x = rt[v];
            const uint32_t w4[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const int r = v * 8 + 2 * k;
              tile[ebase ^ (w4[k] & 0xffffu)] = make_float2(d[r], d[32 + r]);
              tile[ebase ^ (w4[k] >> 16)] = make_float2(d[r + 1], d[32 + r + 1]);
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncthreads();
      if (*flag) {
        bad = true;
        break;
      }
      ph_b ^= 1u;
      ph_mma ^= 1u;
    }
    if (bad) break;

    // store
    {
      const uint64_t gb = tile_base(t, tmask) | my_off;
#pragma unroll 8
      for (int i = 0; i < kPairsPerThread; i++) {
        const float4 v = *reinterpret_cast<const float4*>(tile + (my_sw0 ^ tsw((uint32_t)i * 2u * kFThreads)));
        __stcs(reinterpret_cast<float4*>(amp + (gb | hidep[i])), v);
      }
    }
    __syncthreads();  // the tile buffer is free for the next load
  }

  // leave no async copy or MMA in flight
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (bad && tid == 0) {  // flag bit 1: operand copy pending; bit 2: MMAs pending
    atomicExch(err, 1);
    const int f = *flag;
    if (f & 1) mbar_wait_bounded(bar_b, ph_b);
    if (f & 2) {
      mbar_wait_bounded(bar_mma, ph_mma);
      mbar_wait_bounded(bar_mma + 8, ph_mma);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

int launch_fused_pass(void* amp, int n, const FusedPassDev& pass, const FusedBlockDev* d_blocks,
                      const uint8_t* d_images, int* d_err, int num_sms, cudaStream_t stream) {
  if (n < 13 || pass.num_blocks == 0 || pass.num_blocks > (uint32_t)kMaxBlocks ||
      pass.num_low < 1 || pass.num_low + pass.num_high != 13)
    return MLB_ERR_INVALID_ARG;
  static std::atomic<uint64_t> attr_set_mask{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(attr_set_mask.load(std::memory_order_acquire) & bit)) {
    cudaFuncSetAttribute(k_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    attr_set_mask.fetch_or(bit, std::memory_order_release);
  }
  uint64_t grid = (uint64_t)num_sms * 2;  // two CTAs per SM
  if (grid > pass.num_tiles) grid = pass.num_tiles;
  k_fused<<<(unsigned)grid, kFThreads, kSmemBytes, stream>>>(reinterpret_cast<float2*>(amp), pass, d_blocks,
                                                             d_images, d_err);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb
