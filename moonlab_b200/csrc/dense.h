// dense.h -- host side of the dense complex128 segments (mode 2 of the tile
// kernel, kernels_tile.cu).
//
// A register segment of a complex128 tile pass (planner.h) runs dense when it
// fits: four register qubits in a 12-qubit tile, and at most kDenseMaxCond
// conditioning qubits outside them (controls and diagonal keys of its ops,
// tile-local or outside the tile).  Its ops are multiplied into one 16x16
// complex matrix per value of the conditioning qubits, in FP64, by applying
// the ops in turn to the identity (row operations on all 16 columns at once)
// with exactly the semantics of the register-group code (kernels_tile.cu:
// op_pair, op_swap, op_diag and the tile predicates).  The kernel applies
// U = R + iJ with three real products (Gauss's complex multiplication):
//   t1 = R xr,  t2 = J xi,  t3 = (R + J)(xr + xi),
//   yr = t1 - t2,  yi = t3 - t1 - t2,
// 48 FP64 multiply-adds per amplitude instead of the 64 of the real 32x32
// form.  R and J are written in the A-fragment order of mma.sync m8n8k4 f64
// (row.col), R first:
//   fragment (p, i, s), p = 0 (R) or 1 (J), i = 0..1, s = 0..3:
//   lane l holds M[8 i + (l >> 2)][4 s + (l & 3)],
//   row = output slot, column = input slot
// (fragment slots are the register qubits in a chosen order, see below), so
// a lane's B operands are four whole input slots (re, im) and its D results
// two whole output slots (one 16-byte shared-memory access each); R + J is
// formed in registers.  Host-only.
#pragma once

#include <cstring>
#include <utility>
#include <vector>

#include "mlb_internal.h"

namespace mlb {
namespace dense {

inline int popc32(uint32_t x) { return __builtin_popcount(x); }
inline int popc64(uint64_t x) { return __builtin_popcountll(x); }

// Conditioning qubits of a segment outside its register set: tile-local
// (local bit mask) and outside the tile (global bit mask).  False when the
// segment cannot run dense.
inline bool conditioning(const DevSegment& sg, const DevOp* ops, uint32_t& condloc, uint64_t& condout) {
  if (sg.mode != 0 || sg.nbits != 4) return false;
  uint32_t reg = 0;
  for (int b = 0; b < 4; b++) reg |= 1u << sg.bits[b];
  condloc = 0;
  condout = 0;
  for (int o = sg.op_begin; o < sg.op_end; o++) {
    const DevOp& d = ops[o];
    switch (d.kind) {
      case DOP_1Q_GEN:
      case DOP_1Q_REAL:
      case DOP_X:
      case DOP_SWAP: break;
      case DOP_DIAG1:
        if (d.lt >= 0) condloc |= 1u << d.lt;
        break;
      case DOP_PHASE:
      case DOP_ZZ: condloc |= d.lmask; break;
      default: return false;
    }
    condloc |= d.lcmask;
    condout |= d.ocmask | d.omask;
  }
  condloc &= ~reg;
  return popc32(condloc) <= kDenseMaxCondLoc && popc64(condout) <= kDenseMaxCondOut &&
         popc32(condloc) + popc64(condout) <= kDenseMaxCond;
}

// One op applied to the segment matrix U (U[out][in] over the 16 slots in
// sg.bits order, real and imaginary parts apart) from the left: the op acts
// on every column at once.  locs[k]: the tile-local bits of slot k (the
// variant's conditioning local bits included); tb: the variant's outside
// bits (global).
inline void apply_rows(const DevOp& d, const uint32_t* locs, uint64_t tb, double (*Ur)[16], double (*Ui)[16]) {
  if ((tb & d.ocmask) != d.ocmask) return;  // outside controls (tile predicate)
  if (d.kind == DOP_PHASE && (tb & d.omask) != d.omask) return;
  const double m0r = d.m[0], m0i = d.m[1], m1r = d.m[2], m1i = d.m[3];
  const double m2r = d.m[4], m2i = d.m[5], m3r = d.m[6], m3i = d.m[7];
  auto ctrl_ok = [&](int k) { return (locs[k] & d.lcmask) == d.lcmask; };
  auto scale = [&](int k, double pr, double pi) {
    for (int c = 0; c < 16; c++) {
      const double xr = Ur[k][c], xi = Ui[k][c];
      Ur[k][c] = pr * xr - pi * xi;
      Ui[k][c] = pr * xi + pi * xr;
    }
  };
  switch (d.kind) {
    case DOP_1Q_GEN:
    case DOP_1Q_REAL:
    case DOP_X: {
      const int bt = 1 << d.rt;
      for (int k = 0; k < 16; k++) {
        if ((k & bt) || !ctrl_ok(k)) continue;
        double* r0 = Ur[k];
        double* i0 = Ui[k];
        double* r1 = Ur[k | bt];
        double* i1 = Ui[k | bt];
        if (d.kind == DOP_X) {
          for (int c = 0; c < 16; c++) {
            std::swap(r0[c], r1[c]);
            std::swap(i0[c], i1[c]);
          }
          continue;
        }
        for (int c = 0; c < 16; c++) {
          const double ar = r0[c], ai = i0[c], br = r1[c], bi = i1[c];
          r0[c] = m0r * ar - m0i * ai + m1r * br - m1i * bi;
          i0[c] = m0r * ai + m0i * ar + m1r * bi + m1i * br;
          r1[c] = m2r * ar - m2i * ai + m3r * br - m3i * bi;
          i1[c] = m2r * ai + m2i * ar + m3r * bi + m3i * br;
        }
      }
      break;
    }
    case DOP_SWAP: {
      const int b0 = 1 << d.rt, b1 = 1 << d.rt2;
      for (int k = 0; k < 16; k++) {
        if ((k & (b0 | b1)) || !ctrl_ok(k)) continue;
        for (int c = 0; c < 16; c++) {
          std::swap(Ur[k | b0][c], Ur[k | b1][c]);
          std::swap(Ui[k | b0][c], Ui[k | b1][c]);
        }
      }
      break;
    }
    case DOP_DIAG1:
    case DOP_ZZ: {
      int la = 31, lb = 31;
      if (d.kind == DOP_DIAG1) {
        if (d.lt >= 0) la = d.lt;
      } else {
        uint32_t lm = d.lmask;
        if (lm) { la = __builtin_ctz(lm); lm &= lm - 1; }
        if (lm) lb = __builtin_ctz(lm);
      }
      const uint32_t tkey = (uint32_t)(popc64(tb & d.omask) & 1);
      for (int k = 0; k < 16; k++) {
        if (!ctrl_ok(k)) continue;
        const uint32_t l = locs[k];
        const uint32_t key = ((l >> la) ^ (l >> lb) ^ tkey) & 1u;
        if (key) scale(k, m1r, m1i);
        else scale(k, m0r, m0i);
      }
      break;
    }
    case DOP_PHASE:
      for (int k = 0; k < 16; k++)
        if ((locs[k] & d.lmask) == d.lmask) scale(k, m0r, m0i);
      break;
    default: break;
  }
}

// Per-segment data that the fragment fill needs besides the segment itself.
struct SegPlan {
  int locbits[kDenseMaxCondLoc];
  int kappa[16];  // fragment slot -> matrix slot (register qubits in sg.bits order)
  int nvar;
};

// Tables of one segment of pass P (everything but the matrices).  False when
// the segment does not fit.
inline bool plan_segment(const DevPass& P, const DevSegment& sg, const DevOp* ops, DenseSegDev& D, SegPlan& S) {
  uint32_t cl = 0;
  uint64_t co = 0;
  if (P.L + P.H != kTileBitsC128 || !conditioning(sg, ops, cl, co)) return false;
  std::memset(&D, 0, sizeof D);
  uint32_t reg = 0;
  for (int b = 0; b < 4; b++) reg |= 1u << sg.bits[b];
  int nloc = 0, nout = 0;
  for (int b = 0; b < kTileBitsC128; b++)
    if (cl >> b & 1u) S.locbits[nloc++] = b;
  for (int b = 0; b < 64; b++)
    if (co >> b & 1ull) D.obit[nout++] = (uint8_t)b;
  D.nloc = (uint8_t)nloc;
  D.nout = (uint8_t)nout;
  S.nvar = 1 << (nloc + nout);

  // Bank groups: a 16-byte access lands in bank group = low 3 bits of
  // tile_swz16(e), to which tile bit p adds bit p mod 3.  An 8-lane phase of
  // the B loads varies fragment slot bits 0, 1 and group bit 0; one of the D
  // stores varies slot bit 0 and group bits 1, 2.  Choose the slot order
  // (fragment slot bit i = register qubit perm[i]) and the first three group
  // bits so that those bits reach distinct bank-group bits.
  auto ub = [](int p) { return p >= 0 ? 1 << (p % 3) : 0; };
  int perm[4] = {0, 1, 2, 3};
  bool found = false;
  for (int i = 0; i < 4 && !found; i++)
    for (int j = i + 1; j < 4 && !found; j++)
      if (ub(sg.bits[i]) != ub(sg.bits[j])) {
        int rest = 2;
        perm[0] = i;
        perm[1] = j;
        for (int k = 0; k < 4; k++)
          if (k != i && k != j) perm[rest++] = k;
        found = true;
      }
  // group-index bits: three chosen free bits, the other free local bits, then
  // the conditioning ones (a run of 8 groups shares its conditioning values)
  int free_bits[kDenseGroupBits], nfree = 0;
  for (int b = 0; b < kTileBitsC128; b++)
    if (!(reg >> b & 1u) && !(cl >> b & 1u)) free_bits[nfree++] = b;
  bool used[kDenseGroupBits] = {};
  auto pick = [&](int avoid) {  // a free bit whose bank-group bit is outside `avoid`
    for (int i = 0; i < nfree; i++)
      if (!used[i] && !(ub(free_bits[i]) & avoid)) { used[i] = true; return free_bits[i]; }
    for (int i = 0; i < nfree; i++)
      if (!used[i]) { used[i] = true; return free_bits[i]; }
    return -1;  // not reached: at least 4 free bits
  };
  const int u0 = ub(sg.bits[perm[0]]), u1 = ub(sg.bits[perm[1]]);
  int gbits[kDenseGroupBits];
  gbits[0] = pick(u0 | u1);
  gbits[1] = pick(u0);
  gbits[2] = pick(u0 | ub(gbits[1]));
  int ng = 3;
  for (int i = 0; i < nfree; i++)
    if (!used[i]) gbits[ng++] = free_bits[i];
  for (int i = 0; i < nloc; i++) gbits[ng++] = S.locbits[i];

  for (int c = 0; c < 8; c++) {
    uint32_t e = 0;
    for (int i = 0; i < 3; i++)
      if (c >> i & 1) e |= 1u << gbits[i];
    D.g_lo[c] = (uint16_t)tile_swz16(e);
  }
  for (int h = 0; h < (1 << kDenseColBits); h++) {
    uint32_t e = 0;
    for (int i = 0; i < kDenseColBits; i++)
      if (h >> i & 1) e |= 1u << gbits[3 + i];
    D.g_hi[h] = (uint16_t)tile_swz16(e);
  }
  for (int a = 0; a < 16; a++) {
    uint32_t e = 0;
    S.kappa[a] = 0;
    for (int i = 0; i < 4; i++)
      if (a >> i & 1) {
        e |= 1u << sg.bits[perm[i]];
        S.kappa[a] |= 1 << perm[i];
      }
    D.amp_off[a] = (uint16_t)tile_swz16(e);
  }
  return true;
}

// The matrices of a planned segment: S.nvar variants of kDenseVarDoubles
// doubles at out.
inline void fill_fragments(const DevSegment& sg, const DevOp* ops, const DenseSegDev& D, const SegPlan& S,
                           double* out) {
  // the ops before the first one that reads a conditioning bit are the same
  // for every variant: their product is computed once
  uint32_t locmask = 0;
  uint64_t outmask = 0;
  for (int i = 0; i < D.nloc; i++) locmask |= 1u << S.locbits[i];
  for (int j = 0; j < D.nout; j++) outmask |= 1ull << D.obit[j];
  int first_dep = sg.op_begin;
  for (; first_dep < sg.op_end; first_dep++) {
    const DevOp& d = ops[first_dep];
    uint32_t keys = d.lcmask;
    if (d.kind == DOP_PHASE || d.kind == DOP_ZZ) keys |= d.lmask;
    if (d.kind == DOP_DIAG1 && d.lt >= 0) keys |= 1u << d.lt;
    if ((keys & locmask) || ((d.ocmask | d.omask) & outmask)) break;
  }
  uint32_t slot_loc[16];  // tile-local bits of each slot (register bits only)
  for (int k = 0; k < 16; k++) {
    slot_loc[k] = 0;
    for (int b = 0; b < 4; b++)
      if (k >> b & 1) slot_loc[k] |= 1u << sg.bits[b];
  }
  double Pr[16][16], Pi[16][16];  // U[out][in] over the matrix slots: the common prefix
  for (int k = 0; k < 16; k++)
    for (int c = 0; c < 16; c++) {
      Pr[k][c] = k == c ? 1.0 : 0.0;
      Pi[k][c] = 0.0;
    }
  for (int o = sg.op_begin; o < first_dep; o++) apply_rows(ops[o], slot_loc, 0, Pr, Pi);
  for (int v = 0; v < S.nvar; v++) {
    uint32_t locv = 0;
    uint64_t tb = 0;
    for (int i = 0; i < D.nloc; i++)
      if (v >> i & 1) locv |= 1u << S.locbits[i];
    for (int j = 0; j < D.nout; j++)
      if (v >> (D.nloc + j) & 1) tb |= 1ull << D.obit[j];
    uint32_t locs[16];  // tile-local bits of each slot under this variant
    for (int k = 0; k < 16; k++) locs[k] = slot_loc[k] | locv;
    double Ur[16][16], Ui[16][16];
    std::memcpy(Ur, Pr, sizeof Ur);
    std::memcpy(Ui, Pi, sizeof Ui);
    for (int o = first_dep; o < sg.op_end; o++) apply_rows(ops[o], locs, tb, Ur, Ui);
    double* f = out + (size_t)v * kDenseVarDoubles;
    for (int p = 0; p < 2; p++)
      for (int i = 0; i < 2; i++)
        for (int sk = 0; sk < 4; sk++)
          for (int l = 0; l < 32; l++) {
            const int ao = 8 * i + (l >> 2), ai = 4 * sk + (l & 3);
            const double* row = p == 0 ? Ur[S.kappa[ao]] : Ui[S.kappa[ao]];
            f[((p * 2 + i) * 4 + sk) * 32 + l] = row[S.kappa[ai]];
          }
  }
}

// Dense form of one segment of pass P: appends its dense segment and
// fragments and returns true, or returns false (appending nothing).
inline bool build_segment(const DevPass& P, const DevSegment& sg, const DevOp* ops,
                          std::vector<DenseSegDev>& dsegs, std::vector<double>& frags) {
  DenseSegDev D;
  SegPlan S;
  if (!plan_segment(P, sg, ops, D, S)) return false;
  D.frag_off = (uint32_t)frags.size();
  frags.resize(frags.size() + (size_t)S.nvar * kDenseVarDoubles);
  fill_fragments(sg, ops, D, S, frags.data() + D.frag_off);
  dsegs.push_back(D);
  return true;
}

}  // namespace dense
}  // namespace mlb
