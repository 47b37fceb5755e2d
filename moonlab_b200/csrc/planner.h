// planner.h -- groups a gate-op sequence into tile passes and, inside a
// pass, into register-group segments (used by the state engine and by the
// adjoint-gradient engine).  Host-only.
#pragma once

#include <algorithm>
#include <iterator>
#include <cstdint>
#include <cstring>
#include <vector>

#include "mlb_internal.h"

namespace mlb {
namespace plan {

inline int popc(uint64_t x) { return __builtin_popcountll(x); }

// Tile geometry per dtype (must match TileCfg in kernels_tile.cu).
struct Geo {
  int TB, RB;
};
inline Geo geo(int dtype) { return dtype == MLB_C128 ? Geo{kTileBitsC128, 4} : Geo{13, 4}; }

// Non-diagonal target qubits of an op (must lie inside a tile) and all the
// qubits it touches (targets, controls, diagonal keys).
inline uint64_t op_targets(const mlb_op_t& o) {
  switch (o.kind) {
    case MLB_OP_1Q:
    case MLB_OP_X: return 1ull << o.target;
    case MLB_OP_2Q:
    case MLB_OP_SWAP: return (1ull << o.target) | (1ull << o.target2);
    default: return 0;  // diagonal
  }
}
inline uint64_t op_qubits(const mlb_op_t& o) {
  uint64_t q = o.cmask | op_targets(o);
  if (o.kind == MLB_OP_DIAG1) q |= 1ull << o.target;
  if (o.kind == MLB_OP_ZZ) q |= (1ull << o.target) | (1ull << o.target2);
  return q;
}

// ---------------------------------------------------------------------------
// planner
// ---------------------------------------------------------------------------
struct PlannedPass {
  DevPass pass;
  int seg_begin, seg_end;
};

struct Planner {
  uint32_t n;
  int dtype;
  Geo g;
  int max_ops = kMaxPassOps;  // ops per pass (the op program lives in shared memory)
  // complex128 with dense segments: a register segment is closed before an
  // op that would take its conditioning qubits (controls and diagonal keys
  // outside its four register bits) past what one dense 16x16 segment holds,
  // since a segment over the limit runs gate by gate at several times the
  // cost; a segment is padded with conditioning bits first, and a pass's
  // unused high slots are filled so that every tile has all its bits
  bool dense_limits = false;
  // with dense_limits: a pass's last register segment of at most this many
  // ops goes back to the remaining ops (it would cost a whole dense segment;
  // the next pass usually takes it into one of its segments)
  int defer_tail = 12;
  std::vector<PlannedPass> passes;
  std::vector<DevSegment> segs;
  std::vector<DevOp> dops;
  std::vector<int> dop_src;  // index into the planned ops of every entry of dops

  // Choose the ops of one pass from `rem` (indices into ops), program order.
  // Returns taken indices; fills high mask.
  std::vector<int> choose(const std::vector<mlb_op_t>& ops, const std::vector<int>& rem, int L,
                          uint64_t& SH_out) {
    const uint64_t lowm = (1ull << L) - 1ull;
    const int Hmax = g.TB - L;
    const uint64_t allm = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
    // strategy A: first come
    auto run = [&](uint64_t SH, bool grow, std::vector<int>* taken) {
      uint64_t blocked = 0;
      int cnt = 0;
      for (int idx : rem) {
        const mlb_op_t& o = ops[idx];
        const uint64_t Q = op_qubits(o), T = op_targets(o);
        if (Q & blocked) { blocked |= Q; if (blocked == allm) break; continue; }
        const uint64_t need = T & ~lowm & ~SH;
        if (cnt >= max_ops) break;
        if (need == 0 || (grow && popc(SH | need) <= Hmax)) {
          SH |= need;
          cnt++;
          if (taken) taken->push_back(idx);
        } else {
          blocked |= Q;
          if (blocked == allm) break;
        }
      }
      return std::make_pair(cnt, SH);
    };
    auto A = run(0, true, nullptr);
    // strategy B: the Hmax high qubits most demanded by the first ops
    std::vector<double> score(n, 0.0);
    {
      int seen = 0;
      for (int idx : rem) {
        const uint64_t T = op_targets(ops[idx]) & ~lowm;
        for (uint32_t b = 0; b < n; b++)
          if (T >> b & 1ull) score[b] += 1.0 / (1.0 + seen * 0.02);
        if (++seen > 8 * (int)n) break;
      }
    }
    std::vector<int> order;
    for (uint32_t b = L; b < n; b++) order.push_back((int)b);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return score[a] > score[b]; });
    uint64_t SHB = 0;
    for (int k = 0; k < (int)order.size() && k < Hmax; k++)
      if (score[order[k]] > 0) SHB |= 1ull << order[k];
    auto B = run(SHB, true, nullptr);
    std::vector<int> taken;
    if (B.first > A.first) {
      run(SHB, true, &taken);
      SH_out = B.second;
    } else {
      run(0, true, &taken);
      SH_out = A.second;
    }
    return taken;
  }

  // Reorder a pass's ops (list scheduling) so that ops whose targets fit one
  // register set run back to back: each segment costs a shared-memory round
  // trip of the whole tile, so fewer, fuller segments are cheaper.  Two ops
  // commute when neither's non-diagonal targets touch the other's qubits
  // (controls and diagonal keys commute with each other); an op may only be
  // scheduled once every earlier op it does not commute with is scheduled.
  //
  // `cut` (size N) marks the positions in the returned order where a new
  // segment starts.
  template <typename LocalMask>
  std::vector<int> schedule_segments(const std::vector<mlb_op_t>& ops, const std::vector<int>& taken,
                                     LocalMask&& local_mask, int RB, std::vector<char>& cut) {
    const size_t N = taken.size();
    std::vector<uint32_t> T(N), D(N);
    std::vector<uint64_t> DO(N);
    std::vector<bool> wide(N);
    for (size_t i = 0; i < N; i++) {
      const mlb_op_t& o = ops[taken[i]];
      uint64_t om;
      local_mask(op_targets(o), T[i], om);
      local_mask(op_qubits(o) & ~op_targets(o), D[i], DO[i]);
      wide[i] = o.kind == MLB_OP_2Q;
    }
    // the dense-segment limits for register bits S, local conditioning
    // bits Dl and outside ones Do (padding absorbs up to RB - |S| of Dl)
    auto fits_dense = [&](uint32_t S, uint32_t Dl, uint64_t Do) {
      const int cl = std::max(0, popc(Dl & ~S) - (RB - popc(S)));
      const int co = popc(Do);
      return cl <= kDenseMaxCondLoc && co <= kDenseMaxCondOut && cl + co <= kDenseMaxCond;
    };
    cut.assign(N, 0);
    std::vector<int> blockers(N, 0);
    std::vector<std::vector<int>> after(N);
    for (size_t i = 0; i < N; i++)
      for (size_t j = 0; j < i; j++) {
        const bool commute = (T[i] & (T[j] | D[j])) == 0 && (T[j] & (T[i] | D[i])) == 0;
        if (!commute) {
          blockers[i]++;
          after[j].push_back((int)i);
        }
      }
    std::vector<bool> done(N, false);
    std::vector<int> out;
    out.reserve(N);
    auto take = [&](size_t i) {
      done[i] = true;
      out.push_back(taken[i]);
      for (int k : after[i]) blockers[k]--;
    };
    while (out.size() < N) {
      cut[out.size()] = 1;
      uint32_t S = 0, Dl = 0;
      uint64_t Do = 0;
      bool any = false;
      bool progress = true;
      while (progress) {
        progress = false;
        for (size_t i = 0; i < N; i++) {
          if (done[i] || blockers[i] != 0) continue;
          if (wide[i]) {  // a generic 4x4 op forms its own segment
            if (!any) {
              take(i);
              any = true;
              progress = false;
              break;
            }
            continue;
          }
          if (popc(S | T[i]) <= RB && (!dense_limits || !any || fits_dense(S | T[i], Dl | D[i], Do | DO[i]))) {
            S |= T[i];
            Dl |= D[i];
            Do |= DO[i];
            take(i);
            any = true;
            progress = true;
          }
        }
        if (any && !out.empty() && ops[out.back()].kind == MLB_OP_2Q) break;
      }
    }
    return out;
  }

  template <typename LocalMask>
  std::vector<int> schedule_segments(const std::vector<mlb_op_t>& ops, const std::vector<int>& taken,
                                     LocalMask&& local_mask, int RB) {
    std::vector<char> cut;
    return schedule_segments(ops, taken, local_mask, RB, cut);
  }

  void lower_pass(const std::vector<mlb_op_t>& ops, const std::vector<int>& taken, int L, uint64_t SH) {
    PlannedPass pp{};
    DevPass& P = pp.pass;
    P.n = (int)n;
    P.L = L;
    int local_of[64];
    for (int q = 0; q < 64; q++) local_of[q] = -1;
    for (int q = 0; q < L; q++) local_of[q] = q;
    int H = 0;
    for (uint32_t q = L; q < n; q++)
      if (SH >> q & 1ull) {
        P.high[H] = (int)q;
        local_of[q] = L + H;
        H++;
      }
    P.H = H;
    const int m = L + H;
    const uint64_t allm = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
    P.tile_free_mask = allm & ~(((1ull << L) - 1ull) | SH);
    P.num_tiles = 1ull << (n - m);
    const int RB = std::min(g.RB, m);
    pp.seg_begin = (int)segs.size();

    auto local_mask = [&](uint64_t gm, uint32_t& lm, uint64_t& om) {
      lm = 0;
      om = 0;
      for (uint32_t b = 0; b < n; b++)
        if (gm >> b & 1ull) {
          if (local_of[b] >= 0) lm |= 1u << local_of[b];
          else om |= 1ull << b;
        }
    };
    std::vector<char> cut;
    const std::vector<int> order = schedule_segments(ops, taken, local_mask, RB, cut);
    const std::vector<int>& taken_in = taken;
    (void)taken_in;
    auto run_segments = [&](const std::vector<int>& taken) {
    size_t i = 0;
    while (i < taken.size()) {
      // a generic 4x4 op runs alone in a shared-memory segment
      if (ops[taken[i]].kind == MLB_OP_2Q) {
        const mlb_op_t& o = ops[taken[i]];
        DevSegment sg{};
        sg.mode = 1;
        sg.nbits = 0;
        sg.op_begin = (int)dops.size();
        DevOp d{};
        std::memcpy(d.m, o.m, sizeof d.m);
        local_mask(o.cmask, d.lcmask, d.ocmask);
        d.kind = DOP_2Q_GEN;
        d.lt = local_of[o.target];
        d.k = local_of[o.target2];
        dops.push_back(d);
        dop_src.push_back(taken[i]);
        sg.op_end = (int)dops.size();
        segs.push_back(sg);
        i++;
        continue;
      }
      // grow a segment
      uint32_t bits = 0;
      size_t j = i;
      for (; j < taken.size(); j++) {
        if (ops[taken[j]].kind == MLB_OP_2Q) break;
        if (dense_limits && j > i && cut[j]) break;
        const uint64_t T = op_targets(ops[taken[j]]);
        uint32_t tl = 0;
        uint64_t dummy;
        local_mask(T, tl, dummy);
        if (popc(bits | tl) > RB) break;
        bits |= tl;
      }
      // pad to RB bits: conditioning bits first (dense segments), then the
      // lowest free local bits
      if (dense_limits) {
        uint32_t cond = 0;
        for (size_t k = i; k < j; k++) {
          const mlb_op_t& o = ops[taken[k]];
          uint32_t lm;
          uint64_t om;
          local_mask(op_qubits(o) & ~op_targets(o), lm, om);
          cond |= lm;
        }
        cond &= ~bits;
        for (int b = 0; b < m && popc(bits) < RB; b++)
          if (cond >> b & 1u) bits |= 1u << b;
      }
      for (int b = 0; b < m && popc(bits) < RB; b++) bits |= 1u << b;
      DevSegment sg{};
      sg.nbits = 0;
      for (int b = 0; b < m; b++)
        if (bits >> b & 1u) sg.bits[sg.nbits++] = b;
      auto rpos = [&](int lbit) {
        for (int k = 0; k < sg.nbits; k++)
          if (sg.bits[k] == lbit) return k;
        return -1;
      };
      sg.op_begin = (int)dops.size();
      for (size_t k = i; k < j; k++) {
        const mlb_op_t& o = ops[taken[k]];
        DevOp d{};
        std::memcpy(d.m, o.m, sizeof d.m);
        local_mask(o.cmask, d.lcmask, d.ocmask);
        d.lt = -1;
        switch (o.kind) {
          case MLB_OP_1Q: {
            bool real = true;
            for (int t = 1; t < 8; t += 2)
              if (o.m[t] != 0.0) real = false;
            d.kind = real ? DOP_1Q_REAL : DOP_1Q_GEN;
            d.rt = rpos(local_of[o.target]);
            break;
          }
          case MLB_OP_X: d.kind = DOP_X; d.rt = rpos(local_of[o.target]); break;
          case MLB_OP_SWAP:
            d.kind = DOP_SWAP;
            d.rt = rpos(local_of[o.target]);
            d.rt2 = rpos(local_of[o.target2]);
            break;
          case MLB_OP_DIAG1:
            d.kind = DOP_DIAG1;
            d.lt = local_of[o.target];
            d.omask = d.lt >= 0 ? 0 : (1ull << o.target);
            break;
          case MLB_OP_PHASE: {
            d.kind = DOP_PHASE;
            local_mask(o.cmask, d.lmask, d.omask);
            d.lcmask = 0;
            d.ocmask = 0;
            break;
          }
          case MLB_OP_ZZ: {
            d.kind = DOP_ZZ;
            local_mask((1ull << o.target) | (1ull << o.target2), d.lmask, d.omask);
            break;
          }
        }
        dops.push_back(d);
        dop_src.push_back(taken[k]);
      }
      sg.op_end = (int)dops.size();
      segs.push_back(sg);
      i = j;
    }
    };
    run_segments(order);
    pp.seg_end = (int)segs.size();
    P.num_segments = pp.seg_end - pp.seg_begin;
    passes.push_back(pp);
  }

  void plan(const std::vector<mlb_op_t>& ops) {
    std::vector<int> rem(ops.size());
    for (size_t i = 0; i < ops.size(); i++) rem[i] = (int)i;
    // contiguous low qubits of every tile: complex128 keeps 2 (64-byte rows,
    // two 32-byte sectors; more room for the high qubits the ops need: the
    // 30-qubit depth-40 circuit takes 45 passes of 12-bit tiles, against 55
    // with 3 low qubits), complex64 5
    const int L = (int)n <= g.TB ? (int)n : (dtype == MLB_C128 ? kLowBitsC128 : 5);
    while (!rem.empty()) {
      uint64_t SH = 0;
      std::vector<int> taken;
      if ((int)n <= g.TB) {
        taken.assign(rem.begin(), rem.begin() + std::min<size_t>(rem.size(), kMaxPassOps));
      } else {
        taken = choose(ops, rem, L, SH);
        if (dense_limits) {
          // fill the unused high slots, qubits that condition the pass's
          // ops first (inside the tile, a segment can take them as
          // register bits), then the lowest free ones
          const int Hmax = g.TB - L;
          const uint64_t inside = SH | ((1ull << L) - 1ull);
          std::vector<int> cnt(n, 0);
          for (int idx : taken) {
            const uint64_t q = op_qubits(ops[idx]) & ~inside;
            for (uint32_t b = 0; b < n; b++)
              if (q >> b & 1ull) cnt[b]++;
          }
          std::vector<int> order;
          for (uint32_t b = L; b < n; b++)
            if (!(inside >> b & 1ull)) order.push_back((int)b);
          std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cnt[a] > cnt[b]; });
          for (int k = 0; k < (int)order.size() && popc(SH) < Hmax; k++) SH |= 1ull << order[k];
        }
      }
      lower_pass(ops, taken, L, SH);
      if (dense_limits && defer_tail > 0 && (int)n > g.TB) {
        PlannedPass& pp = passes.back();
        const DevSegment& last = segs[pp.seg_end - 1];
        const int nlast = last.op_end - last.op_begin;
        if (pp.pass.num_segments >= 2 && last.mode == 0 && nlast <= defer_tail) {
          // the last segment's ops were scheduled after every other op of the
          // pass (they depend on or commute with all of them), so running
          // them after the whole pass keeps the circuit
          std::vector<int> back(dop_src.begin() + last.op_begin, dop_src.end());
          std::sort(back.begin(), back.end());
          dops.resize(last.op_begin);
          dop_src.resize(last.op_begin);
          segs.pop_back();
          pp.seg_end--;
          pp.pass.num_segments--;
          std::vector<int> kept;
          std::set_difference(taken.begin(), taken.end(), back.begin(), back.end(), std::back_inserter(kept));
          taken.swap(kept);
        }
      }
      // remove taken (both lists ascending)
      std::vector<int> next;
      next.reserve(rem.size() - taken.size());
      size_t t = 0;
      for (int idx : rem) {
        if (t < taken.size() && taken[t] == idx) { t++; continue; }
        next.push_back(idx);
      }
      rem.swap(next);
    }
  }
};


}  // namespace plan
}  // namespace mlb
