// dense.h -- host side of the dense complex128 segments (mode 2 of the tile
// kernel, kernels_tile.cu).
//
// A register segment of a complex128 tile pass (planner.h) runs dense when it
// fits: four register qubits in a 13-qubit tile, and at most kDenseMaxCond
// conditioning qubits outside them (controls and diagonal keys of its ops,
// tile-local or outside the tile).  Its ops are multiplied into one 16x16
// complex matrix per value of the conditioning qubits, in FP64, by applying
// the ops to the 16 basis vectors with exactly the semantics of the
// register-group code (kernels_tile.cu: op_pair, op_swap, op_diag and the tile
// predicates), and the real 32x32 form of each matrix is written in the
// A-fragment order of mma.sync m8n8k4 f64 (row.col):
//   fragment (i, s), lane l holds A[8 i + (l >> 2)][4 s + (l & 3)],
//   real row 8 i + r  = component i & 1 (re, im) of output slot 8 (i >> 1) + r,
//   real col 4 s + q  = component s & 1 of input slot 4 (s >> 1) + q,
// (fragment slots are the register qubits in a chosen order, see below)
// so a lane's B operands are the re and im parts of four whole input slots
// and its D results the re and im parts of two whole output slots (one
// 16-byte shared-memory access each).  Host-only.
#pragma once

#include <complex>
#include <cstring>
#include <utility>
#include <vector>

#include "mlb_internal.h"

namespace mlb {
namespace dense {

using cd = std::complex<double>;

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

// One op applied to a 16-slot vector x (slots in sg.bits order); locv: the
// conditioning local bits' values (a local mask), tb: the conditioning
// outside bits' values (global).
inline void apply(const DevOp& d, const DevSegment& sg, uint32_t locv, uint64_t tb, cd* x) {
  if ((tb & d.ocmask) != d.ocmask) return;  // outside controls (tile predicate)
  if (d.kind == DOP_PHASE && (tb & d.omask) != d.omask) return;
  auto loc = [&](int k) {
    uint32_t r = locv;
    for (int b = 0; b < 4; b++)
      if (k >> b & 1) r |= 1u << sg.bits[b];
    return r;
  };
  auto ctrl_ok = [&](int k) { return (loc(k) & d.lcmask) == d.lcmask; };
  const cd m0(d.m[0], d.m[1]), m1(d.m[2], d.m[3]), m2(d.m[4], d.m[5]), m3(d.m[6], d.m[7]);
  switch (d.kind) {
    case DOP_1Q_GEN:
    case DOP_1Q_REAL:
    case DOP_X: {
      const int bt = 1 << d.rt;
      for (int k = 0; k < 16; k++) {
        if (k & bt) continue;
        if (!ctrl_ok(k)) continue;
        const cd a0 = x[k], a1 = x[k | bt];
        if (d.kind == DOP_X) {
          x[k] = a1;
          x[k | bt] = a0;
        } else {
          x[k] = m0 * a0 + m1 * a1;
          x[k | bt] = m2 * a0 + m3 * a1;
        }
      }
      break;
    }
    case DOP_SWAP: {
      const int b0 = 1 << d.rt, b1 = 1 << d.rt2;
      for (int k = 0; k < 16; k++) {
        if (k & (b0 | b1)) continue;
        if (!ctrl_ok(k)) continue;
        std::swap(x[k | b0], x[k | b1]);
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
        const uint32_t l = loc(k);
        const uint32_t key = ((l >> la) ^ (l >> lb) ^ tkey) & 1u;
        x[k] *= key ? m1 : m0;
      }
      break;
    }
    case DOP_PHASE:
      for (int k = 0; k < 16; k++)
        if ((loc(k) & d.lmask) == d.lmask) x[k] *= m0;
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
  if (P.L + P.H != 13 || !conditioning(sg, ops, cl, co)) return false;
  std::memset(&D, 0, sizeof D);
  uint32_t reg = 0;
  for (int b = 0; b < 4; b++) reg |= 1u << sg.bits[b];
  int nloc = 0, nout = 0;
  for (int b = 0; b < 13; b++)
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
  int free_bits[9], nfree = 0;
  for (int b = 0; b < 13; b++)
    if (!(reg >> b & 1u) && !(cl >> b & 1u)) free_bits[nfree++] = b;
  bool used[9] = {false, false, false, false, false, false, false, false, false};
  auto pick = [&](int avoid) {  // a free bit whose bank-group bit is outside `avoid`
    for (int i = 0; i < nfree; i++)
      if (!used[i] && !(ub(free_bits[i]) & avoid)) { used[i] = true; return free_bits[i]; }
    for (int i = 0; i < nfree; i++)
      if (!used[i]) { used[i] = true; return free_bits[i]; }
    return -1;  // not reached: at least 5 free bits
  };
  const int u0 = ub(sg.bits[perm[0]]), u1 = ub(sg.bits[perm[1]]);
  int gbits[9];
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
  for (int h = 0; h < 64; h++) {
    uint32_t e = 0;
    for (int i = 0; i < 6; i++)
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

// The matrices of a planned segment: S.nvar variants of 1024 doubles at out.
inline void fill_fragments(const DevSegment& sg, const DevOp* ops, const DenseSegDev& D, const SegPlan& S,
                           double* out) {
  for (int v = 0; v < S.nvar; v++) {
    uint32_t locv = 0;
    uint64_t tb = 0;
    for (int i = 0; i < D.nloc; i++)
      if (v >> i & 1) locv |= 1u << S.locbits[i];
    for (int j = 0; j < D.nout; j++)
      if (v >> (D.nloc + j) & 1) tb |= 1ull << D.obit[j];
    cd U[16][16];  // U[out][in], matrix slots
    for (int c = 0; c < 16; c++) {
      cd x[16];
      for (int k = 0; k < 16; k++) x[k] = k == c ? cd(1.0, 0.0) : cd(0.0, 0.0);
      for (int o = sg.op_begin; o < sg.op_end; o++) apply(ops[o], sg, locv, tb, x);
      for (int k = 0; k < 16; k++) U[k][c] = x[k];
    }
    double* f = out + (size_t)v * 1024;
    for (int i = 0; i < 4; i++)
      for (int sk = 0; sk < 8; sk++)
        for (int l = 0; l < 32; l++) {
          const int ao = 8 * (i >> 1) + (l >> 2), co_ = i & 1;
          const int ai = 4 * (sk >> 1) + (l & 3), ci = sk & 1;
          const cd u = U[S.kappa[ao]][S.kappa[ai]];
          f[(i * 8 + sk) * 32 + l] = co_ == 0 ? (ci == 0 ? u.real() : -u.imag()) : (ci == 0 ? u.imag() : u.real());
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
  frags.resize(frags.size() + (size_t)S.nvar * 1024);
  fill_fragments(sg, ops, D, S, frags.data() + D.frag_off);
  dsegs.push_back(D);
  return true;
}

}  // namespace dense
}  // namespace mlb
