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
// per 128-row half one thread issues that half's MMAs and commits them to
// the half's mbarrier, and after the commit arrives the half's warps read
// their 32 accumulator lanes back (tcgen05.ld 32x32b) into the FP32 tile.
//
// Occupancy: a CTA of 8 warps (warp w owns tensor-memory lane quadrant w & 3
// of half w >> 2, one tile row per thread) holds one tile buffer, two
// operand images (110 KiB of shared memory) and 256 TMEM columns, so two CTAs share an SM: one
// CTA's MMA waits and tile loads (16-byte async copies, cp.async) overlap
// the other's operand conversion and readback.  A tile's loads are issued
// from the previous tile's store loop, into the slots just stored, so they
// overlap the stores.  A half's MMAs start as soon as its own four warps
// have stored their rows (a named barrier per half), and the two halves are
// issued from different SM sub-partitions: one thread issues an MMA only
// every ~70 cycles, so one issuer alone would leave the tensor core half idle
// at N = 64.  MMA descriptors are precomputed (the per-MMA part is a
// constant add).  Each block's operand image comes by one bulk copy
// completing on its buffer's mbarrier; there are two image buffers, and the
// image two applications ahead is requested as soon as both halves' MMAs of
// the current one have completed, so a copy has a whole block's conversion,
// MMAs and readback to land.
//
// Waits are bounded: if one runs out the kernel sets *err, waits once more
// (bounded) for what it issued, frees its tensor memory and returns.
#include <atomic>

#include <cuda_bf16.h>

#include "kernels_common.cuh"
#include "mlb_internal.h"

namespace mlb {

namespace {

constexpr int kFThreads = 256;       // 8 warps: warp w owns TMEM lane quadrant w & 3 of half w >> 2
constexpr int kTileAmps = 1 << 13;
constexpr int kPairsPerThread = kTileAmps / 2 / kFThreads;  // 16
// shared-memory layout (bytes from a 1024-byte aligned base); two CTAs per SM
constexpr uint32_t kBHi = 0;          // operand image buffer 0: 64 rows x 128 B, then lo
constexpr uint32_t kBLo = 8192;
constexpr uint32_t kBImg = 16384;     // buffer 1 at kBImg (two images in flight)
constexpr uint32_t kTile0 = 32768;    // one tile buffer of 2^13 float2 (64 KiB)
constexpr uint32_t kMbarMma = 98304;  // two: one per 128-row half
constexpr uint32_t kMbarB = 98320;    // two: one per image buffer
constexpr uint32_t kTmemSlot = 98336;
constexpr uint32_t kFlag = 98340;
constexpr uint32_t kIssued = 98344;   // two uint32: image copies issued into each buffer
constexpr int kMaxBlocks = 64;        // blocks per pass (the planner splits longer passes)
constexpr uint32_t kColTab = 98352;   // per block: 32 swizzled column offsets (uint32)
constexpr uint32_t kRowTab = kColTab + kMaxBlocks * 128;  // per block: 2 x 16 swizzled row-nibble offsets (uint16)
constexpr uint32_t kHiDep = kRowTab + kMaxBlocks * 64;    // 16 x uint64: global offsets of tile bits 9..12
constexpr uint32_t kImgTab = kHiDep + kPairsPerThread * 8;  // per block: operand image index (uint32)
constexpr int kTbNibbles = 6;         // tile index bits (<= 34 - 13) in nibbles
constexpr uint32_t kTbTab = kImgTab + kMaxBlocks * 4;  // 6 x 16 uint64: tile-index nibble -> global bits
constexpr uint32_t kSmemUsed = kTbTab + kTbNibbles * 16 * 8;
constexpr uint32_t kSmemBytes = kSmemUsed + 1024;  // alignment slack
static_assert(kTile0 >= 2 * kBImg && kMbarMma == kTile0 + 65536 && kColTab >= kIssued + 8, "layout overlap");
static_assert(kColTab % 16 == 0 && kHiDep % 8 == 0 && kTbTab % 8 == 0, "table alignment");
static_assert(2 * (kSmemBytes + 1024) <= 228 * 1024, "two CTAs per SM (1 KiB reserved per CTA)");
constexpr uint32_t kTmemCols = 256;  // D: columns 0..127 (64 per half); A: 128..255
constexpr uint32_t kACol = 128;      // A of half h: hi at kACol + 64 h, lo at kACol + 64 h + 32
constexpr long long kWaitLimit = 1ll << 24;       // try_wait rounds before giving up (a backstop)
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // and 2 s of wall time
constexpr uint64_t kTestWaitLimitNs = 20000000ull;  // 20 ms in the bounded-wait test mode
constexpr uint32_t kWaitHintNs = 100000;          // suspend-time hint of one try_wait

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

// 8 consecutive columns of this thread's lane.
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n" ::"r"(taddr), "r"(v[0]),
               "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

// 16 consecutive columns of this thread's lane (completion: tcgen05.wait::ld).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t* r = reinterpret_cast<uint32_t*>(v);
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

// One try_wait with a suspend-time hint: a thread whose phase has not
// completed sleeps (up to the hint) until it completes instead of spinning,
// so waiting lanes do not take issue slots from the warps that work.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t"
      ".reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(kWaitHintNs)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded by time: false after limit_ns without the phase completing.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (long long i = 0; i < kWaitLimit; i++) {
    if (mbar_try(bar, parity)) return true;
    if (globaltimer_ns() - t0 > limit_ns) return false;
  }
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

// XOR swizzle of the FP32 tile on bits 1..4 (pairs of amplitudes stay
// together, so 16-byte async copies land whole): spreads rows of any stride
// over the banks.
__device__ __forceinline__ uint32_t tsw(uint32_t e) { return e ^ ((((e >> 5) ^ (e >> 9)) & 15u) << 1); }

// Bits 0..nb-1 of v placed at tile bits pos[0..nb-1].
template <int NB>
__device__ __forceinline__ uint32_t deposit(uint32_t v, const uint8_t* pos) {
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < NB; i++) r |= ((v >> i) & 1u) << pos[i];
  return r;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Global bits of tile t: the bits of t placed, in order, at the set bits of
// tmask (the qubits outside the tile), by a 16-entry table per nibble of t.
__device__ __forceinline__ uint64_t tile_base(uint64_t t, const uint64_t* tbtab) {
  uint64_t g = 0;
#pragma unroll
  for (int k = 0; k < kTbNibbles; k++) g |= tbtab[16 * k + ((t >> (4 * k)) & 15u)];
  return g;
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

// test_skip_copy: CTA 0 does not request its first operand image (and waits
// give up after kTestWaitLimitNs), so its first block's waits run out with no
// copy and no MMA in flight -- the bounded-wait test of mlb_test_fused_skip_copy.
__global__ void __launch_bounds__(kFThreads, 2)
    k_fused(float2* __restrict__ amp, FusedPassDev pass, const FusedBlockDev* __restrict__ blocks,
            const uint8_t* __restrict__ images, int* __restrict__ err, int test_skip_copy) {
  const uint64_t wait_ns = test_skip_copy ? kTestWaitLimitNs : kWaitLimitNs;
  extern __shared__ uint8_t smraw[];
  // 1024-byte alignment by pointer arithmetic on the shared array (not
  // through an integer cast), so every access below stays a shared-memory
  // access with 32-bit addressing instead of a generic one
  uint8_t* sm = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
  const uint32_t sbase = smem_u32(sm);
  volatile int* flag = reinterpret_cast<volatile int*>(sm + kFlag);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t half = (uint32_t)warp >> 2, qd = (uint32_t)warp & 3u;  // row m = tid = 128 half + 32 qd + lane
  // bar_mma + 8 h: MMAs of half h done; bar_b + 8 j: operand image in buffer j landed
  const uint32_t bar_mma = sbase + kMbarMma, bar_b = sbase + kMbarB;
  volatile uint32_t* issued = reinterpret_cast<volatile uint32_t*>(sm + kIssued);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + kTmemSlot),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_mma), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_mma + 8), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_b), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_b + 8), "r"(1));
    issued[0] = 0;
    issued[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *flag = 0;
  }

  // Per-block tables, swizzled once (tsw is linear over GF(2), so the offset
  // of tile row m and column r is rowtab(m & 15) ^ rowtab(16 + (m >> 4)) ^ coltab(r)):
  //   coltab: the 32 block columns r (block bits pos[0..4]);
  //   rowtab: the 16 values of each nibble of m (tile bits q[0..3], q[4..7]).
  uint32_t* coltab = reinterpret_cast<uint32_t*>(sm + kColTab);
  uint16_t* rowtab = reinterpret_cast<uint16_t*>(sm + kRowTab);
  uint32_t* imgtab = reinterpret_cast<uint32_t*>(sm + kImgTab);
  for (uint32_t i = tid; i < pass.num_blocks * 32u; i += kFThreads) {
    const FusedBlockDev blk = blocks[pass.block_begin + i / 32u];
    const uint32_t j = i & 31u;
    coltab[i] = tsw(deposit<5>(j, blk.pos));
    rowtab[i] = (uint16_t)tsw(j < 16 ? deposit<4>(j, blk.q) : deposit<4>(j - 16u, blk.q + 4));
    if (j == 0) imgtab[i / 32u] = blk.image;
  }
  if (tid < kPairsPerThread)
    reinterpret_cast<uint64_t*>(sm + kHiDep)[tid] = tile_global(0, (uint32_t)tid * 2u * kFThreads, pass);
  uint64_t hmask = (1ull << pass.num_low) - 1ull;
#pragma unroll
  for (int i = 0; i < 12; i++)
    if (i < (int)pass.num_high) hmask |= 1ull << pass.hbits[i];
  uint64_t* tbtab = reinterpret_cast<uint64_t*>(sm + kTbTab);
  if (tid < kTbNibbles * 16) {  // entry (k, v): bits of v at set bits 4k .. 4k+3 of the free bits
    const int k = tid >> 4;
    const uint32_t v = (uint32_t)tid & 15u;
    uint64_t m = (pass.free_mask >> 63) ? (pass.free_mask & ~(1ull << 63)) : ~hmask, g = 0;
    for (int j = 0; j < 4 * k && m; j++) m &= m - 1;
    for (int i = 0; i < 4 && m; i++) {
      if (v >> i & 1u) g |= m & (~m + 1);
      m &= m - 1;
    }
    tbtab[tid] = g;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kTmemSlot);


  // Tile-local index e of this thread's i-th amplitude pair: e = 512 i + 2 tid.
  // Its global offset is linear in e over disjoint bits, so it splits into
  // a per-thread part (bits 0..8) and a per-i part (bits 9..12, shared table).
  const uint64_t my_off = tile_global(0, 2u * (uint32_t)tid, pass);
  const uint64_t* hidep = reinterpret_cast<const uint64_t*>(sm + kHiDep);
  // tsw(512 i + 2 tid) = tsw(512 i) ^ tsw(2 tid), the first term a
  // compile-time constant in the unrolled loops
  const uint32_t my_sw0 = tsw(2u * (uint32_t)tid);
  // this thread's lane quadrant in tensor memory
  const uint32_t tlane = tmem + ((qd * 32u) << 16);
  // operand-image descriptor; the start-address field (bits 0..13, address >> 4)
  // of the other K chunks and of the lo image is this plus a constant (the
  // shared window is below 256 KiB, so the field does not carry)
  const uint64_t desc_b = sdesc(sbase + kBHi);

  // Block applications s = 0, 1, ... of this CTA (tile by tile, block by
  // block) take operand buffer s & 1; application s + 2's image is requested
  // as soon as application s's MMAs have completed.
  uint32_t ph_mma = 0, s = 0;
  bool bad = false;
  // operand image of block b for tile t (per-vector image sets: the tile's
  // vector picks its set)
  auto image_of = [&](uint64_t t, uint32_t b) -> const uint8_t* {
    return images + ((size_t)imgtab[b] + (size_t)(t >> pass.vec_shift) * pass.vec_images) * 16384;
  };
  if (tid == 0) {
    const uint32_t nb = pass.num_blocks;
    if ((uint64_t)blockIdx.x < pass.num_tiles && !(test_skip_copy && blockIdx.x == 0)) {
      issued[0] = 1;
      bulk_load(sbase + kBHi, image_of(blockIdx.x, 0), 16384, bar_b);
    }
    const uint64_t t1 = (uint64_t)blockIdx.x + (nb > 1 ? 0ull : (uint64_t)gridDim.x);
    if (t1 < pass.num_tiles) {
      issued[1] = 1;
      bulk_load(sbase + kBImg, image_of(t1, nb > 1 ? 1 : 0), 16384, bar_b + 8);
    }
  }
  float2* tile = reinterpret_cast<float2*>(sm + kTile0);
  // A tile's loads are issued by the previous tile's store loop (each thread
  // refills the 16-byte slots it has just stored), except for the first tile.
  bool prefetched = false;
  for (uint64_t t = blockIdx.x; t < pass.num_tiles && !bad; t += gridDim.x) {
    if (!prefetched) {
      const uint64_t gb = tile_base(t, tbtab) | my_off;
      const uint32_t dst0 = sbase + kTile0;
#pragma unroll 8
      for (int i = 0; i < kPairsPerThread; i++)
        cp_async16(dst0 + (my_sw0 ^ tsw((uint32_t)i * 2u * kFThreads)) * 8u, amp + (gb | hidep[i]));
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();

    for (uint32_t b = 0; b < pass.num_blocks; b++) {
      const uint32_t ebase = rowtab[b * 32u + (tid & 15)] ^ rowtab[b * 32u + 16u + ((uint32_t)tid >> 4)];
      const uint4* ct = reinterpret_cast<const uint4*>(coltab + b * 32u);
      // When tile bit 0 is the block's lowest bit, columns 2k and 2k + 1 are
      // adjacent amplitudes (offsets differ in bit 0 only; the swizzle keeps
      // pairs together): move each pair as one 16-byte access.  Otherwise all
      // of a warp's rows would hit one bank pair per column (tile bit 0 is
      // the only bit that sets a float2's half of its 16-byte bank group).
      const bool pairs = (coltab[b * 32u] ^ coltab[b * 32u + 1u]) == 1u;
      // Amplitude operand, row m = tid, in two groups of 16 columns r: word j
      // holds K elements 2j, 2j+1 (re of r for K < 32, im of r - 32 above),
      // hi and lo parts; group g fills words 8g..8g+7 of each quarter.
      {
        const uint32_t ta = tlane + kACol + half * 64u;
#pragma unroll
        for (int g = 0; g < 2; g++) {
          uint32_t hre[8], him[8], lre[8], lim[8];
#pragma unroll
          for (int c = 0; c < 4; c++) {  // columns 16 g + 4 c .. + 3
            const uint4 o = ct[4 * g + c];
            float2 a0, a1, a2, a3;
            if (pairs) {  // block-uniform
              const float4 p0 = *reinterpret_cast<const float4*>(tile + (ebase ^ o.x));
              const float4 p1 = *reinterpret_cast<const float4*>(tile + (ebase ^ o.z));
              a0 = make_float2(p0.x, p0.y);
              a1 = make_float2(p0.z, p0.w);
              a2 = make_float2(p1.x, p1.y);
              a3 = make_float2(p1.z, p1.w);
            } else {
              a0 = tile[ebase ^ o.x];
              a1 = tile[ebase ^ o.y];
              a2 = tile[ebase ^ o.z];
              a3 = tile[ebase ^ o.w];
            }
            const __nv_bfloat162 h0 = __floats2bfloat162_rn(a0.x, a1.x), h1 = __floats2bfloat162_rn(a0.y, a1.y);
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(a2.x, a3.x), h3 = __floats2bfloat162_rn(a2.y, a3.y);
            const float2 f0 = __bfloat1622float2(h0), f1 = __bfloat1622float2(h1);
            const float2 f2 = __bfloat1622float2(h2), f3 = __bfloat1622float2(h3);
            hre[2 * c] = *reinterpret_cast<const uint32_t*>(&h0);
            him[2 * c] = *reinterpret_cast<const uint32_t*>(&h1);
            hre[2 * c + 1] = *reinterpret_cast<const uint32_t*>(&h2);
            him[2 * c + 1] = *reinterpret_cast<const uint32_t*>(&h3);
            lre[2 * c] = pack_bf16x2(a0.x - f0.x, a1.x - f0.y);
            lim[2 * c] = pack_bf16x2(a0.y - f1.x, a1.y - f1.y);
            lre[2 * c + 1] = pack_bf16x2(a2.x - f2.x, a3.x - f2.y);
            lim[2 * c + 1] = pack_bf16x2(a2.y - f3.x, a3.y - f3.y);
          }
          tmem_st8(ta + 8u * g, hre);
          tmem_st8(ta + 16u + 8u * g, him);
          tmem_st8(ta + 32u + 8u * g, lre);
          tmem_st8(ta + 48u + 8u * g, lim);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      }
      // Each half's MMAs start once its four warps have stored their rows
      // (named barrier 1 + half) and are issued by one thread of that half,
      // on different SM sub-partitions (warps 0 and 5), so the two halves'
      // MMA streams overlap.
      if (half == 0) asm volatile("bar.sync 1, 128;\n" ::: "memory");
      else asm volatile("bar.sync 2, 128;\n" ::: "memory");
      if (tid == 0 || tid == 160) {
        const uint32_t buf = s & 1u;
        if (mbar_wait_bounded(bar_b + 8u * buf, (s >> 1) & 1u, wait_ns)) {  // operand image landed
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t a_h = tmem + kACol + half * 64u, d_h = tmem + half * 64u;
#pragma unroll
          for (int kc = 0; kc < 3; kc++) {
#pragma unroll
            for (int kk = 0; kk < 4; kk++)
              mma_bf16_ts(d_h, a_h + (kc == 1 ? 32u : 0u) + kk * 8u,
                          desc_b + (uint64_t)((buf * kBImg + (kc == 2 ? kBLo : kBHi) + kk * 32u) >> 4),
                          (kc | kk) != 0 ? 1u : 0u);
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                           bar_mma + 8u * half)
                       : "memory");
        } else {
          atomicOr((int*)flag, 1);  // operand copy not seen; this half's MMAs not issued
        }
      }
      // Readback of this warp's 32 accumulator lanes of its half; warp 5 also
      // waits for half 0 and then requests the next operand image.
      {
        int ok = 0;
        __syncwarp();
        if (lane == 0 && !*flag) {
          ok = mbar_wait_bounded(bar_mma + 8u * half, ph_mma, wait_ns) ? 1 : 0;
          if (ok && warp == 5) ok = mbar_wait_bounded(bar_mma, ph_mma, wait_ns) ? 1 : 0;  // and half 0
          if (!ok) atomicOr((int*)flag, 2);
          if (ok && warp == 5) {  // buffer s & 1 is free: application s + 2's image into it
            const uint32_t r = b + 2u, adv = r / pass.num_blocks, buf = s & 1u;
            const uint64_t t2 = t + (uint64_t)adv * gridDim.x;
            if (t2 < pass.num_tiles) {
              issued[buf] = issued[buf] + 1u;
              bulk_load(sbase + buf * kBImg, image_of(t2, r % pass.num_blocks), 16384, bar_b + 8u * buf);
            }
          }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok) {
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t td = tlane + half * 64u;
#pragma unroll
          for (int g = 0; g < 2; g++) {  // columns r = 16 g .. 16 g + 15
            float dre[16], dim[16];
            tmem_ld16(td + 16u * g, dre);
            tmem_ld16(td + 32u + 16u * g, dim);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int c = 0; c < 4; c++) {
              const uint4 o = ct[4 * g + c];
              if (pairs) {
                *reinterpret_cast<float4*>(tile + (ebase ^ o.x)) =
                    make_float4(dre[4 * c], dim[4 * c], dre[4 * c + 1], dim[4 * c + 1]);
                *reinterpret_cast<float4*>(tile + (ebase ^ o.z)) =
                    make_float4(dre[4 * c + 2], dim[4 * c + 2], dre[4 * c + 3], dim[4 * c + 3]);
              } else {
                tile[ebase ^ o.x] = make_float2(dre[4 * c], dim[4 * c]);
                tile[ebase ^ o.y] = make_float2(dre[4 * c + 1], dim[4 * c + 1]);
                tile[ebase ^ o.z] = make_float2(dre[4 * c + 2], dim[4 * c + 2]);
                tile[ebase ^ o.w] = make_float2(dre[4 * c + 3], dim[4 * c + 3]);
              }
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      // every thread that sets the flag reads it back here, so all agree
      if (__syncthreads_or(*flag != 0)) {
        bad = true;
        break;
      }
      s++;
      ph_mma ^= 1u;
    }
    if (bad) break;

    // store, and the next tile's loads into the slots just read (this
    // thread's own slots, read before: no barrier needed in between)
    {
      const uint64_t gb = tile_base(t, tbtab) | my_off;
      const uint64_t next = t + gridDim.x;
      prefetched = next < pass.num_tiles;
      const uint64_t ngb = prefetched ? (tile_base(next, tbtab) | my_off) : 0;
      const uint32_t dst0 = sbase + kTile0;
#pragma unroll 8
      for (int i = 0; i < kPairsPerThread; i++) {
        const uint32_t slot = my_sw0 ^ tsw((uint32_t)i * 2u * kFThreads);
        const float4 v = *reinterpret_cast<const float4*>(tile + slot);
        __stcs(reinterpret_cast<float4*>(amp + (gb | hidep[i])), v);  // consumes v: the slot has been read
        if (prefetched) cp_async16(dst0 + slot * 8u, amp + (ngb | hidep[i]));
      }
      if (prefetched) asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    __syncthreads();
  }

  // leave no async copy or MMA in flight
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (bad && tid == 0) {
    atomicExch(err, 1);
    // the last image copy issued into each buffer may be pending (at most one
    // per buffer: a buffer is refilled only after its previous image was used)
    for (uint32_t j = 0; j < 2; j++)
      if (issued[j]) mbar_wait_bounded(bar_b + 8u * j, (issued[j] - 1u) & 1u, wait_ns);
    // either half's MMAs may be in flight (the halves have separate issuers)
    mbar_wait_bounded(bar_mma, ph_mma, wait_ns);
    mbar_wait_bounded(bar_mma + 8, ph_mma, wait_ns);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
}

// One operand image per (block, vector): thread c builds column c of the
// block's 32x32 unitary in FP64 (the gates applied in order to basis vector
// c, as the adjoint's forward passes apply them: RY = [[c, -s], [s, c]],
// RZ = diag(c - i s, c + i s), X / CNOT a swap), then all threads write the
// bf16 hi / lo split of U' in the swizzled K-major layout.
__global__ void __launch_bounds__(128) k_fused_images(const FusedGenBlock* __restrict__ blocks, int num_blocks,
                                                      const FusedGenOp* __restrict__ ops,
                                                      const double2* __restrict__ cs, int num_params,
                                                      uint8_t* __restrict__ images) {
  __shared__ double2 U[32][33];  // U[row][column]
  const int k = blockIdx.x, v = blockIdx.y, tid = threadIdx.x;
  const FusedGenBlock blk = blocks[k];
  if (tid < 32) {
    const int c = tid;
    for (int r = 0; r < 32; r++) U[r][c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    for (uint32_t o = 0; o < blk.num_ops; o++) {
      const FusedGenOp g = ops[blk.op_begin + o];
      const uint32_t tb = 1u << g.lt;
      const uint32_t cm = g.lc >= 0 ? (1u << g.lc) : 0u;
      double2 t = make_double2(1.0, 0.0);
      if (g.kind != ADJ_KIND_X) t = cs[(size_t)v * num_params + g.p];
      for (uint32_t i = 0; i < 32; i++) {
        if ((i & tb) || (i & cm) != cm) continue;
        const double2 a0 = U[i][c], a1 = U[i | tb][c];
        if (g.kind == ADJ_KIND_X) {
          U[i][c] = a1;
          U[i | tb][c] = a0;
        } else if (g.kind == ADJ_KIND_RY) {
          U[i][c] = make_double2(t.x * a0.x - t.y * a1.x, t.x * a0.y - t.y * a1.y);
          U[i | tb][c] = make_double2(t.y * a0.x + t.x * a1.x, t.y * a0.y + t.x * a1.y);
        } else {  // RZ: key 0 -> (c - i s), key 1 -> (c + i s)
          U[i][c] = make_double2(t.x * a0.x + t.y * a0.y, t.x * a0.y - t.y * a0.x);
          U[i | tb][c] = make_double2(t.x * a1.x - t.y * a1.y, t.x * a1.y + t.y * a1.x);
        }
      }
    }
  }
  __syncthreads();
  uint16_t* hi = reinterpret_cast<uint16_t*>(images + ((size_t)v * num_blocks + k) * 16384);
  uint16_t* lo = hi + 4096;
  for (int idx = tid; idx < 64 * 64; idx += blockDim.x) {
    const int rn = idx >> 6, kk = idx & 63;
    const double2 u = U[rn & 31][kk & 31];
    const double x = rn < 32 ? (kk < 32 ? u.x : -u.y) : (kk < 32 ? u.y : u.x);
    const __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    const __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    // element (rn, kk) at byte (rn / 8) * 1024 + (rn % 8) * 128 + 2 kk, 16-byte chunk xor rn % 8
    const uint32_t off = (((uint32_t)(rn >> 3) * 1024u + (uint32_t)(rn & 7) * 128u + 2u * (uint32_t)kk) ^
                          ((uint32_t)(rn & 7) << 4)) >> 1;
    hi[off] = *reinterpret_cast<const uint16_t*>(&h);
    lo[off] = *reinterpret_cast<const uint16_t*>(&l);
  }
}

}  // namespace

int launch_fused_images(const FusedGenBlock* blocks, int num_blocks, const FusedGenOp* ops, const double2* cs,
                        int num_params, int batch, uint8_t* images, cudaStream_t stream) {
  if (num_blocks < 1 || batch < 1 || batch > 65535 || !blocks || !ops || !cs || !images) return MLB_ERR_INVALID_ARG;
  k_fused_images<<<dim3((unsigned)num_blocks, (unsigned)batch), 128, 0, stream>>>(blocks, num_blocks, ops, cs,
                                                                                  num_params, images);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

int launch_fused_pass(void* amp, int n, const FusedPassDev& pass, const FusedBlockDev* d_blocks,
                      const uint8_t* d_images, int* d_err, int num_sms, cudaStream_t stream, int test_skip_copy) {
  // n: bits of the tile enumeration (a batch of B states of N qubits: N +
  // ceil(log2 B)); num_tiles may stop short of 2^(n - 13) (B not a power of 2)
  if (n < 13 || n > 13 + 4 * kTbNibbles || pass.num_blocks == 0 || pass.num_blocks > (uint32_t)kMaxBlocks ||
      pass.num_low < 1 || pass.num_low + pass.num_high != 13 || pass.num_tiles == 0 ||
      pass.num_tiles > 1ull << (n - 13) || pass.vec_shift > 63)
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
                                                             d_images, d_err, test_skip_copy);
  count_launch();
  return cudaGetLastError() == cudaSuccess ? MLB_OK : MLB_ERR_DRIVER;
}

}  // namespace mlb
