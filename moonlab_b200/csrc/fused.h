// fused.h -- host planning of the fused complex64 path: gates are grouped
// into dense blocks of k <= 5 qubits, blocks into tile passes, and each
// block's 32x32 unitary is written as the tensor-core operand the fused
// kernel reads (kernels_fused.cu).
//
// Block building is greedy with look-ahead over the gate order: a block
// takes the earliest unplaced op, then every later op whose qubits (targets
// and controls) keep the block within 5 qubits, as long as no earlier
// unplaced op shares a qubit with it (that op would have to act first).
// k = 1 blocks of a single qubit are the 1q-run fusion of fusion.c:247-292;
// here runs of 1- and 2-qubit gates on up to 5 qubits collapse into one
// 2^5 x 2^5 complex matrix.
//
// A tile pass holds the 4 low qubits (128-byte contiguous runs) and 9 chosen
// high qubits (2^13 amplitudes, 64 KiB of complex64).  Blocks on fewer than 5 qubits are
// padded with other tile qubits (identity on them).
//
// Operand: for a block U (32x32 complex), the real 64x64 matrix
//   U' = [Re U  -Im U; Im U  Re U]   (rows: outputs (re 0..31, im 32..63),
//                                     cols: inputs  (re 0..31, im 32..63))
// split as U' = hi + lo with hi = bf16(U'), lo = bf16(U' - hi), each stored
// in the tensor core's K-major 128-byte-swizzled layout: element (n, k) at
// byte (n / 8) * 1024 + (n % 8) * 128 + 2 k, with the 16-byte chunk index
// XORed with n % 8.  8 KiB per half, 16 KiB per block.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "moonlab_b200.h"
#include "mlb_internal.h"
#include "planner.h"

namespace mlb {
namespace fused {

constexpr int kTileBits = 13;     // 2^13 complex64 amplitudes per tile
constexpr int kLowBits = 4;       // 16 contiguous amplitudes (128 B) per tile row
constexpr int kHighBits = kTileBits - kLowBits;
constexpr int kBlockQubits = 5;
constexpr size_t kBImageBytes = 16384;  // hi (8 KiB) + lo (8 KiB)
constexpr size_t kMaxPassBlocks = 64;   // blocks per launch (the kernel's offset tables)

using cd = std::complex<double>;

struct Block {
  uint64_t qmask = 0;
  std::vector<int> ops;  // indices into the op list, in application order
};

struct PassPlan {
  uint64_t hmask = 0;           // the high tile qubits
  std::vector<int> blocks;      // indices into the block list
};

struct Plan {
  std::vector<Block> blocks;
  std::vector<PassPlan> passes;
  std::vector<FusedBlockDev> dev_blocks;  // in pass order
  std::vector<FusedPassDev> dev_passes;
  std::vector<uint8_t> images;            // kBImageBytes per dev block
};

// Apply op o to a 2^k local vector; lb[q] = local bit of global qubit q.
inline void apply_local(cd* v, int k, const mlb_op_t& o, const int* lb) {
  const uint32_t dim = 1u << k;
  uint32_t cm = 0;
  for (int q = 0; q < 64; q++)
    if (o.cmask >> q & 1ull) cm |= 1u << lb[q];
  auto M = [&](int idx) { return cd(o.m[2 * idx], o.m[2 * idx + 1]); };
  switch (o.kind) {
    case MLB_OP_1Q:
    case MLB_OP_X:
    case MLB_OP_DIAG1: {
      const uint32_t tb = 1u << lb[o.target];
      for (uint32_t i = 0; i < dim; i++) {
        if ((i & tb) || (i & cm) != cm) continue;
        const cd a0 = v[i], a1 = v[i | tb];
        if (o.kind == MLB_OP_X) {
          v[i] = a1;
          v[i | tb] = a0;
        } else if (o.kind == MLB_OP_DIAG1) {
          v[i] = M(0) * a0;
          v[i | tb] = M(1) * a1;
        } else {
          v[i] = M(0) * a0 + M(1) * a1;
          v[i | tb] = M(2) * a0 + M(3) * a1;
        }
      }
      return;
    }
    case MLB_OP_2Q: {
      const uint32_t b0 = 1u << lb[o.target], b1 = 1u << lb[o.target2];
      for (uint32_t i = 0; i < dim; i++) {
        if ((i & (b0 | b1)) || (i & cm) != cm) continue;
        const uint32_t idx[4] = {i, i | b0, i | b1, i | b0 | b1};
        cd x[4], y[4];
        for (int c = 0; c < 4; c++) x[c] = v[idx[c]];
        for (int r = 0; r < 4; r++) {
          y[r] = 0;
          for (int c = 0; c < 4; c++) y[r] += M(r * 4 + c) * x[c];
        }
        for (int c = 0; c < 4; c++) v[idx[c]] = y[c];
      }
      return;
    }
    case MLB_OP_SWAP: {
      const uint32_t b0 = 1u << lb[o.target], b1 = 1u << lb[o.target2];
      for (uint32_t i = 0; i < dim; i++) {
        if ((i & (b0 | b1)) || (i & cm) != cm) continue;
        std::swap(v[i | b0], v[i | b1]);
      }
      return;
    }
    case MLB_OP_ZZ: {
      const uint32_t b0 = 1u << lb[o.target], b1 = 1u << lb[o.target2];
      for (uint32_t i = 0; i < dim; i++) {
        if ((i & cm) != cm) continue;
        const bool same = ((i & b0) != 0) == ((i & b1) != 0);
        v[i] *= same ? M(0) : M(1);
      }
      return;
    }
    case MLB_OP_PHASE: {
      for (uint32_t i = 0; i < dim; i++)
        if ((i & cm) == cm) v[i] *= M(0);
      return;
    }
    default:
      return;
  }
}

inline uint16_t bf16_bits(double x) {
  // round to nearest even on the float value, then to bf16
  float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan
  const uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  return (uint16_t)(u >> 16);
}
inline double bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return (double)f;
}

inline size_t sw128_offset(int row, int k) {  // bf16 element (row, k), 64 per row
  const size_t lin = (size_t)(row / 8) * 1024 + (size_t)(row % 8) * 128 + (size_t)k * 2;
  return lin ^ ((size_t)(row % 8) << 4);
}

// Greedy look-ahead grouping of ops into <= 5-qubit blocks.  Returns
// MLB_ERR_NOT_SUPPORTED if an op spans more than 5 qubits.
inline int make_blocks(const std::vector<mlb_op_t>& ops, uint32_t n, std::vector<Block>& out) {
  const uint64_t all = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
  std::vector<uint64_t> qm(ops.size());
  for (size_t i = 0; i < ops.size(); i++) {
    qm[i] = plan::op_qubits(ops[i]);
    if (plan::popc(qm[i]) > kBlockQubits) return MLB_ERR_NOT_SUPPORTED;
  }
  std::vector<char> placed(ops.size(), 0);
  size_t first = 0;
  out.clear();
  while (first < ops.size()) {
    Block b;
    uint64_t blocked = 0;
    for (size_t i = first; i < ops.size(); i++) {
      if (placed[i]) continue;
      const uint64_t q = qm[i];
      if (q & blocked) {
        blocked |= q;
      } else if (plan::popc(b.qmask | q) <= kBlockQubits) {
        b.qmask |= q;
        b.ops.push_back((int)i);
        placed[i] = 1;
      } else {
        blocked |= q;
      }
      if (blocked == all) break;
    }
    out.push_back(std::move(b));
    while (first < ops.size() && placed[first]) first++;
  }
  return MLB_OK;
}

inline int emit(const std::vector<mlb_op_t>& ops, uint32_t n, Plan& P,
                const std::vector<std::vector<int>>& pass_blocks, const std::vector<uint64_t>& pass_h);

// Group whole blocks into passes (5 low + <= 8 high qubits) and emit the
// device program and operand images.
inline int plan_passes(const std::vector<mlb_op_t>& ops, uint32_t n, Plan& P) {
  if (n < (uint32_t)kTileBits) return MLB_ERR_NOT_SUPPORTED;
  const uint64_t all = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
  const uint64_t low = (1ull << kLowBits) - 1ull;
  std::vector<char> placed(P.blocks.size(), 0);
  size_t first = 0;
  P.passes.clear();
  while (first < P.blocks.size()) {
    PassPlan pp;
    uint64_t blocked = 0;
    for (size_t j = first; j < P.blocks.size(); j++) {
      if (placed[j]) continue;
      const uint64_t q = P.blocks[j].qmask;
      if (q & blocked) {
        blocked |= q;
      } else if (plan::popc(pp.hmask | (q & ~low)) <= kHighBits) {
        pp.hmask |= q & ~low;
        pp.blocks.push_back((int)j);
        placed[j] = 1;
      } else {
        blocked |= q;
      }
      if (blocked == all) break;
    }
    P.passes.push_back(std::move(pp));
    while (first < P.blocks.size() && placed[first]) first++;
  }
  std::vector<std::vector<int>> pb;
  std::vector<uint64_t> ph;
  for (auto& pp : P.passes) {
    pb.push_back(pp.blocks);
    ph.push_back(pp.hmask);
  }
  return emit(ops, n, P, pb, ph);
}

// Device program and operand images for passes (block lists, high masks);
// each pass is padded to exactly 8 high qubits.
inline int emit(const std::vector<mlb_op_t>& ops, uint32_t n, Plan& P,
                const std::vector<std::vector<int>>& pass_blocks, const std::vector<uint64_t>& pass_h) {
  P.passes.clear();
  for (size_t i = 0; i < pass_blocks.size(); i++) {
    uint64_t h = pass_h[i];
    for (uint32_t g = kLowBits; g < n && plan::popc(h) < kHighBits; g++) h |= 1ull << g;
    // at most kMaxPassBlocks per launch: longer runs become consecutive passes on the same tile
    for (size_t b0 = 0; b0 < pass_blocks[i].size(); b0 += kMaxPassBlocks) {
      PassPlan pp;
      pp.hmask = h;
      const size_t b1 = std::min(pass_blocks[i].size(), b0 + kMaxPassBlocks);
      pp.blocks.assign(pass_blocks[i].begin() + b0, pass_blocks[i].begin() + b1);
      P.passes.push_back(std::move(pp));
    }
  }
  // device program
  P.dev_blocks.clear();
  P.dev_passes.clear();
  P.images.clear();
  for (const auto& pp : P.passes) {
    FusedPassDev dp{};
    dp.num_low = (uint8_t)kLowBits;
    dp.num_high = (uint8_t)kHighBits;
    int tile_pos[64];
    for (int g = 0; g < 64; g++) tile_pos[g] = -1;
    for (int g = 0; g < kLowBits; g++) tile_pos[g] = g;
    int h = 0;
    for (uint32_t g = kLowBits; g < n; g++)
      if (pp.hmask >> g & 1ull) {
        dp.hbits[h] = (uint8_t)g;
        tile_pos[g] = kLowBits + h;
        h++;
      }
    dp.num_tiles = 1ull << (n - kTileBits);
    dp.vec_shift = 63;
    dp.vec_images = 0;
    dp.block_begin = (uint32_t)P.dev_blocks.size();
    dp.num_blocks = (uint32_t)pp.blocks.size();
    for (int bi : pp.blocks) {
      const Block& B = P.blocks[bi];
      // block bits: its qubits by tile position, padded with unused tile positions
      std::vector<int> pos;
      for (uint32_t g = 0; g < n; g++)
        if (B.qmask >> g & 1ull) pos.push_back(tile_pos[g]);
      std::sort(pos.begin(), pos.end());
      for (int t = 0; t < kTileBits && (int)pos.size() < kBlockQubits; t++)
        if (std::find(pos.begin(), pos.end(), t) == pos.end()) pos.push_back(t);
      std::sort(pos.begin(), pos.end());
      FusedBlockDev db{};
      std::vector<int> rows;  // the tile bits outside the block: a thread's row index m
      for (int t = 0; t < kTileBits; t++) {
        const auto it = std::find(pos.begin(), pos.end(), t);
        if (it != pos.end()) db.pos[it - pos.begin()] = (uint8_t)t;
        else rows.push_back(t);
      }
      // Row bits 0..3 are the lanes of one shared-memory phase (16 lanes of
      // 8-byte accesses; 8 lanes of 16-byte pair accesses when tile bit 0 is
      // the block's first column bit).  Under the kernel's tile swizzle, tile
      // bit t moves a float2's bank-pair index (bits 0..3) along bit
      // class(t): t = 0 -> 0; t = 1, 5, 9 -> 1; 2, 6, 10 -> 2; 3, 7, 11 -> 3;
      // 4, 8, 12 -> none.  Putting one row bit of each class first makes the
      // phase's lanes hit distinct banks.
      {
        auto cls = [](int t) { return t == 0 ? 0 : (t % 4 == 0) ? -1 : (t - 1) % 4 + 1; };
        const bool pairs = pos[0] == 0;
        std::vector<int> order;
        for (int want = pairs ? 1 : 0; want <= 3; want++)
          for (int t : rows)
            if (cls(t) == want && std::find(order.begin(), order.end(), t) == order.end()) {
              order.push_back(t);
              break;
            }
        for (int t : rows)
          if (std::find(order.begin(), order.end(), t) == order.end()) order.push_back(t);
        for (int i = 0; i < (int)order.size(); i++) db.q[i] = (uint8_t)order[i];
      }
      // local bit of each global qubit: the index of its tile position in pos
      int lb[64];
      for (int g = 0; g < 64; g++) lb[g] = 0;
      for (uint32_t g = 0; g < n; g++)
        if (tile_pos[g] >= 0) {
          const auto it = std::find(pos.begin(), pos.end(), tile_pos[g]);
          if (it != pos.end()) lb[g] = (int)(it - pos.begin());
        }
      // U column by column
      std::vector<cd> U(32 * 32);
      cd v[32];
      for (int c = 0; c < 32; c++) {
        for (int r = 0; r < 32; r++) v[r] = (r == c) ? 1.0 : 0.0;
        for (int oi : B.ops) apply_local(v, kBlockQubits, ops[oi], lb);
        for (int r = 0; r < 32; r++) U[r * 32 + c] = v[r];
      }
      // operand image: U' rows n (outputs), columns k (inputs), hi then lo
      const size_t off = P.images.size();
      P.images.resize(off + kBImageBytes);
      uint8_t* hi = P.images.data() + off;
      uint8_t* lo = hi + kBImageBytes / 2;
      for (int rn = 0; rn < 64; rn++)
        for (int k = 0; k < 64; k++) {
          const cd u = U[(rn & 31) * 32 + (k & 31)];
          double x;
          if (rn < 32) x = k < 32 ? u.real() : -u.imag();
          else x = k < 32 ? u.imag() : u.real();
          const uint16_t h16 = bf16_bits(x);
          const uint16_t l16 = bf16_bits(x - bf16_value(h16));
          std::memcpy(hi + sw128_offset(rn, k), &h16, 2);
          std::memcpy(lo + sw128_offset(rn, k), &l16, 2);
        }
      db.image = (uint32_t)(off / kBImageBytes);
      P.dev_blocks.push_back(db);
    }
    P.dev_passes.push_back(dp);
  }
  return MLB_OK;
}

// Pass-first planning: choose each pass's tile over the ops (every qubit of
// an op, controls included, inside the tile; greedy look-ahead in op order),
// then fuse the pass's ops into blocks on the tile's 13 qubits.  Ops are
// finer than blocks, so passes pack more work than grouping whole blocks.
inline int plan(const std::vector<mlb_op_t>& ops, uint32_t n, Plan& P) {
  if (n < (uint32_t)kTileBits) return MLB_ERR_NOT_SUPPORTED;
  const uint64_t all = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
  const uint64_t low = (1ull << kLowBits) - 1ull;
  std::vector<uint64_t> qm(ops.size());
  for (size_t i = 0; i < ops.size(); i++) {
    qm[i] = plan::op_qubits(ops[i]);
    if (plan::popc(qm[i]) > kBlockQubits) return MLB_ERR_NOT_SUPPORTED;
  }
  std::vector<char> placed(ops.size(), 0);
  size_t first = 0;
  P.blocks.clear();
  std::vector<std::vector<int>> pass_blocks;
  std::vector<uint64_t> pass_h;
  // One pass from the unplaced ops, in order: an op joins if all its qubits
  // fit the tile (growing the high set up to 8 when `grow`) and no skipped
  // op shares a qubit with it.
  auto run = [&](uint64_t hmask, bool grow, std::vector<int>* taken) {
    uint64_t blocked = 0;
    int cnt = 0;
    for (size_t i = first; i < ops.size(); i++) {
      if (placed[i]) continue;
      const uint64_t q = qm[i];
      const uint64_t need = q & ~low & ~hmask;
      if (q & blocked) {
        blocked |= q;
      } else if (need == 0 || (grow && plan::popc(hmask | need) <= kHighBits)) {
        hmask |= need;
        cnt++;
        if (taken) taken->push_back((int)i);
      } else {
        blocked |= q;
      }
      if (blocked == all) break;
    }
    return std::make_pair(cnt, hmask);
  };
  while (first < ops.size()) {
    // strategy A: first come; strategy B: the 8 high qubits most used by
    // the next ops (weighted toward the front); keep the one placing more
    const auto A = run(0, true, nullptr);
    std::vector<double> score(n, 0.0);
    int seen = 0;
    for (size_t i = first; i < ops.size() && seen < 8 * (int)n; i++) {
      if (placed[i]) continue;
      const uint64_t q = qm[i] & ~low;
      for (uint32_t b = 0; b < n; b++)
        if (q >> b & 1ull) score[b] += 1.0 / (1.0 + seen * 0.02);
      seen++;
    }
    std::vector<int> order;
    for (uint32_t b = kLowBits; b < n; b++) order.push_back((int)b);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return score[a] > score[b]; });
    uint64_t hb = 0;
    for (int k = 0; k < (int)order.size() && k < kHighBits; k++)
      if (score[order[k]] > 0) hb |= 1ull << order[k];
    const auto Bs = run(hb, true, nullptr);
    std::vector<int> mine;
    const uint64_t hmask = (Bs.first > A.first ? run(hb, true, &mine) : run(0, true, &mine)).second;
    for (int i : mine) placed[i] = 1;
    while (first < ops.size() && placed[first]) first++;
    // blocks over this pass's ops (their order is a valid order of the pass)
    std::vector<mlb_op_t> sub;
    sub.reserve(mine.size());
    for (int i : mine) sub.push_back(ops[i]);
    std::vector<Block> bl;
    int rc = make_blocks(sub, n, bl);
    if (rc) return rc;
    std::vector<int> ids;
    for (auto& b : bl) {
      for (auto& oi : b.ops) oi = mine[oi];  // back to indices into ops
      ids.push_back((int)P.blocks.size());
      P.blocks.push_back(std::move(b));
    }
    pass_blocks.push_back(std::move(ids));
    pass_h.push_back(hmask);
  }
  // reuse plan_passes' emission by presetting the pass list
  return emit(ops, n, P, pass_blocks, pass_h);
}

}  // namespace fused
}  // namespace mlb
