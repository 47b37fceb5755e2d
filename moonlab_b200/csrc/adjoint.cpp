// adjoint.cpp -- host runtime of the batched adjoint gradient for the
// hardware-efficient ansatz (C ABI: mlb_hea_* in include/moonlab_b200.h).
//
// Tape (vqe_build_hea_diff_circuit, vqe.c:1946-1981): X on every set bit of
// hf_reference, then per layer l: for q in 0..N-1: RY(q, theta[2(lN+q)]),
// RZ(q, theta[2(lN+q)+1]); then CNOT(q, q+1) for q in 0..N-2.
//
// One evaluation of B parameter vectors:
//   1. cos/sin(theta/2) table on the host (libm, as gate_ry / gate_rz do);
//   2. psi[b] = |hf>; forward tile passes over the tape;
//   3. lambda = H psi in tile passes over the Pauli terms; the last pass also
//      produces E_b = <psi_b|lambda_b> (per-tile partials, fixed-order sum);
//   4. backward tile passes over the reversed tape on (psi, lambda) with the
//      per-parameter partials of Im<lambda|G|psi>; fixed-order sums.
// Checkpoints: the tape is planned in segments of s = ceil(sqrt(L)) layers.
// The forward sweep keeps psi at every segment boundary, and the backward
// sweep restores psi from them instead of relying on the inverse gates
// across the whole circuit, so the uncompute drift is bounded by one
// segment (C - 1 extra states per vector for C segments).  Memory policy:
// checkpoints when they fit next to the whole batch; when memory is short
// they are dropped first (pure uncompute), then the batch runs in
// sub-batches.  mlb_hea_set_checkpointing overrides the policy.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "fused.h"
#include "mlb_internal.h"
#include "planner.h"

using namespace mlb;
using namespace mlb::plan;

namespace {

thread_local std::string g_herr;
int hfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_herr = buf;
  return code;
}

struct TapeOp {
  int kind;  // ADJ_KIND_X (CNOT when ctrl >= 0), ADJ_KIND_RY, ADJ_KIND_RZ
  int q;
  int ctrl;
  int p;
};

struct GatePass {
  AdjPass P;
  std::vector<AdjOp> ops;
  std::vector<int> param_of_slot;
  size_t ops_off = 0, slots_off = 0;  // offsets into the device arrays
};
struct TermPass {
  AdjPass P;
  std::vector<AdjTerm> terms;
  size_t terms_off = 0;
};

}  // namespace

struct mlb_hea {
  uint32_t n = 0, layers = 0, P = 0;
  uint64_t hf = 0;
  int dtype = MLB_C128, device = 0, num_sms = 148;
  std::vector<uint64_t> xm, zm;
  std::vector<double> coeff;
  std::vector<TapeOp> tape;
  std::vector<GatePass> fwd, bwd;
  // segments: fwd passes [fwd_seg[k], fwd_seg[k+1]) run segment k; bwd
  // passes [bwd_seg[j], bwd_seg[j+1]) run segment C-1-j backwards
  std::vector<size_t> fwd_seg, bwd_seg;
  uint32_t seg_layers = 0;
  int ckpt_mode = 0;         // 0 auto, 1 always, -1 never
  void* ckpt = nullptr;
  size_t ckpt_cap = 0;       // bytes
  int last_ckpt = 0;
  size_t last_chunks = 0;
  std::vector<TermPass> lam;
  cudaStream_t stream = nullptr;
  // device buffers
  void* psi = nullptr;
  void* lamb = nullptr;
  size_t batch_cap = 0;
  double2* d_cs = nullptr;
  size_t cs_cap = 0;
  double* d_part = nullptr;
  size_t part_cap = 0;
  double* d_epart = nullptr;
  size_t epart_cap = 0;
  AdjOp* d_ops = nullptr;
  AdjTerm* d_terms = nullptr;
  int* d_slots = nullptr;
  double* d_out = nullptr;  // [B] energies then [B][P] grads
  size_t out_cap = 0;
  unsigned char* d_gram = nullptr;  // geometry: Gram matrix, then the Gram kernel's scratch
  size_t gram_cap = 0;
  size_t budget = 0;         // bytes for psi + lambda; 0 = 80% of free memory
  // complex64 forward sweep on the tensor cores (N >= 13): per segment, fused
  // passes of <= 5-qubit blocks whose operand images are built on the device
  // per vector from the cos/sin table (k_fused_images)
  int fused_mode = 0;        // 0 auto (complex64, N >= 13), 1 on, -1 off
  bool fused_ok = false;     // the fused plans exist
  int last_fused = 0;
  std::vector<std::vector<FusedPassDev>> fseg;  // per forward segment
  std::vector<FusedBlockDev> fblocks;           // image = the block's index among all segments' blocks
  std::vector<FusedGenBlock> gblocks;
  std::vector<FusedGenOp> gops;
  FusedBlockDev* d_fblocks = nullptr;
  FusedGenBlock* d_gblocks = nullptr;
  FusedGenOp* d_gops = nullptr;
  uint8_t* d_images = nullptr;
  size_t images_cap = 0;     // bytes
  int* d_ferr = nullptr;
  double* d_norm = nullptr;
  size_t norm_cap = 0;
};

namespace {

struct Guard {
  int prev = -1;
  explicit Guard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~Guard() {
    int c = -1;
    cudaGetDevice(&c);
    if (prev >= 0 && c != prev) cudaSetDevice(prev);
  }
};

int cfail(cudaError_t e, const char* what) {
  return hfail(e == cudaErrorMemoryAllocation ? MLB_ERR_OUT_OF_MEMORY : MLB_ERR_DRIVER, "%s: %s", what,
               cudaGetErrorString(e));
}

template <typename T>
int grow(T*& p, size_t& cap, size_t count) {
  if (cap >= count && p) return MLB_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return cfail(e, "adjoint buffer");
  cap = count;
  return MLB_OK;
}

// Proxy engine ops so the state engine's planner can choose tile qubits.
mlb_op_t proxy(const TapeOp& t) {
  mlb_op_t o{};
  o.target2 = -1;
  o.target = t.q;
  if (t.kind == ADJ_KIND_X) {
    o.kind = MLB_OP_X;
    o.cmask = t.ctrl >= 0 ? (1ull << t.ctrl) : 0;
  } else if (t.kind == ADJ_KIND_RY) {
    o.kind = MLB_OP_1Q;
  } else {
    o.kind = MLB_OP_DIAG1;
  }
  return o;
}

// Partition a tape (forward or reversed) into gate passes and lower them.
void plan_gates(mlb_hea* h, const std::vector<TapeOp>& tape, bool backward, std::vector<GatePass>& out) {
  const int TB = adj_tile_bits(h->dtype, backward);
  Planner pl{h->n, h->dtype, Geo{TB, 3}};
  pl.max_ops = std::min({kMaxAdjOps, kMaxAdjSlots, kMaxAdjSegs});
  std::vector<mlb_op_t> px;
  px.reserve(tape.size());
  for (const auto& t : tape) px.push_back(proxy(t));
  const int n = (int)h->n;
  const int L = n <= TB ? n : 5;
  std::vector<int> rem(tape.size());
  for (size_t i = 0; i < tape.size(); i++) rem[i] = (int)i;
  while (!rem.empty()) {
    uint64_t SH = 0;
    std::vector<int> taken;
    if (n <= TB) taken.assign(rem.begin(), rem.begin() + std::min<size_t>(rem.size(), pl.max_ops));
    else taken = pl.choose(px, rem, L, SH);
    GatePass gp{};
    AdjPass& P = gp.P;
    P.n = n;
    P.L = L;
    int local_of[64];
    for (int q = 0; q < 64; q++) local_of[q] = q < L ? q : -1;
    int H = 0;
    for (int q = L; q < n; q++)
      if (SH >> q & 1ull) {
        P.high[H] = q;
        local_of[q] = L + H;
        H++;
      }
    P.H = H;
    const int m = L + H;
    const uint64_t allm = (1ull << n) - 1ull;
    P.tile_free_mask = allm & ~(((1ull << L) - 1ull) | SH);
    P.tiles_per_state = 1ull << (n - m);
    P.num_params = (int)h->P;
    auto local_mask = [&](uint64_t gm, uint32_t& lm, uint64_t& om) {
      lm = 0;
      om = 0;
      for (int b = 0; b < n; b++)
        if (gm >> b & 1ull) {
          if (local_of[b] >= 0) lm |= 1u << local_of[b];
          else om |= 1ull << b;
        }
    };
    const std::vector<int> order = pl.schedule_segments(px, taken, local_mask, 3);
    // pack into segments of <= 3 register bits (padded with the lowest free bits)
    size_t i = 0;
    while (i < order.size()) {
      uint32_t bits = 0;
      size_t j = i;
      for (; j < order.size(); j++) {
        uint32_t tl;
        uint64_t om;
        local_mask(op_targets(px[order[j]]), tl, om);
        if (__builtin_popcount(bits | tl) > 3) break;
        bits |= tl;
      }
      for (int b = 0; b < m && __builtin_popcount(bits) < 3; b++) bits |= 1u << b;
      AdjSeg& sg = P.segs[P.num_segments++];
      int nb = 0;
      for (int b = 0; b < m && nb < 3; b++)
        if (bits >> b & 1u) sg.bits[nb++] = b;
      for (; nb < 3; nb++) sg.bits[nb] = sg.bits[nb - 1];  // never reached for m >= 3
      sg.op_begin = (int)gp.ops.size();
      for (size_t k = i; k < j; k++) {
        const TapeOp& t = tape[order[k]];
        AdjOp a{};
        a.kind = t.kind;
        a.p = t.p;
        a.slot = -1;
        a.lt = -1;
        a.qt = t.q;
        a.rt = 0;
        if (t.kind != ADJ_KIND_RZ) {
          const int lb = local_of[t.q];
          for (int r = 0; r < 3; r++)
            if (sg.bits[r] == lb) a.rt = r;
        } else {
          a.lt = local_of[t.q];
        }
        if (t.ctrl >= 0) {
          uint64_t om;
          local_mask(1ull << t.ctrl, a.lcmask, om);
          a.ocmask = om;
        }
        if (backward && t.p >= 0) {
          a.slot = (int)gp.param_of_slot.size();
          gp.param_of_slot.push_back(t.p);
        }
        gp.ops.push_back(a);
      }
      sg.op_end = (int)gp.ops.size();
      i = j;
    }
    P.num_ops = (int)gp.ops.size();
    P.num_slots = (int)gp.param_of_slot.size();
    out.push_back(std::move(gp));
    std::vector<int> next;
    size_t t = 0;
    for (int idx : rem) {
      if (t < taken.size() && taken[t] == idx) { t++; continue; }
      next.push_back(idx);
    }
    rem.swap(next);
  }
}

// Partition the Pauli terms into lambda passes: a term fits a pass when its
// X-part lies inside the tile (Z-part may lie anywhere).  Terms commute in
// the sum, so no ordering constraint applies.
void plan_terms(mlb_hea* h) {
  const int TB = adj_tile_bits(h->dtype, false);
  const int n = (int)h->n;
  const int L = n <= TB ? n : 5;
  const int Hmax = n <= TB ? 0 : TB - L;
  const uint64_t lowm = (1ull << L) - 1ull;
  std::vector<int> rem(h->xm.size());
  for (size_t i = 0; i < rem.size(); i++) rem[i] = (int)i;
  while (!rem.empty()) {
    uint64_t SH = 0;
    std::vector<int> taken, left;
    for (int t : rem) {
      const uint64_t need = h->xm[t] & ~lowm & ~SH;
      if ((int)taken.size() < kMaxAdjTerms && __builtin_popcountll(SH | need) <= Hmax) {
        SH |= need;
        taken.push_back(t);
      } else {
        left.push_back(t);
      }
    }
    TermPass tp{};
    AdjPass& P = tp.P;
    P.n = n;
    P.L = L;
    int local_of[64];
    for (int q = 0; q < 64; q++) local_of[q] = q < L ? q : -1;
    int H = 0;
    for (int q = L; q < n; q++)
      if (SH >> q & 1ull) {
        P.high[H] = q;
        local_of[q] = L + H;
        H++;
      }
    P.H = H;
    const uint64_t allm = (1ull << n) - 1ull;
    P.tile_free_mask = allm & ~(((1ull << L) - 1ull) | SH);
    P.tiles_per_state = 1ull << (n - L - H);
    for (int t : taken) {
      AdjTerm a{};
      for (int b = 0; b < n; b++) {
        if (h->xm[t] >> b & 1ull) a.xl |= 1u << local_of[b];
        if (h->zm[t] >> b & 1ull) {
          if (local_of[b] >= 0) a.zl |= 1u << local_of[b];
          else a.zo |= 1ull << b;
        }
      }
      const int ny = __builtin_popcountll(h->xm[t] & h->zm[t]) & 3;
      const double c = h->coeff[t];
      a.cr = ny == 0 ? c : ny == 2 ? -c : 0.0;
      a.ci = ny == 1 ? c : ny == 3 ? -c : 0.0;
      tp.terms.push_back(a);
    }
    P.num_ops = (int)tp.terms.size();
    h->lam.push_back(std::move(tp));
    rem.swap(left);
  }
}

// Fused plans of the forward sweep (complex64, N >= 13): each segment's gates
// grouped into <= 5-qubit blocks and tile passes by the fused planner (on
// stand-in ops: only their qubits matter), each block's gates recorded in
// its local qubits for the device image builder.  False when a segment does
// not plan (the CUDA-core forward passes then run).
bool plan_fused_forward(mlb_hea* h, const std::vector<size_t>& cut) {
  const uint32_t n = h->n;
  if (n < (uint32_t)fused::kTileBits) return false;
  for (size_t k = 0; k + 1 < cut.size(); k++) {
    const std::vector<TapeOp> sub(h->tape.begin() + cut[k], h->tape.begin() + cut[k + 1]);
    std::vector<mlb_op_t> ops;
    ops.reserve(sub.size());
    for (const TapeOp& t : sub) ops.push_back(proxy(t));
    fused::Plan P;
    if (fused::plan(ops, n, P) != MLB_OK) return false;
    std::vector<FusedPassDev> passes;
    size_t j = 0;  // P.dev_blocks are in pass order
    for (size_t pi = 0; pi < P.passes.size(); pi++) {
      FusedPassDev dp = P.dev_passes[pi];
      dp.block_begin = (uint32_t)h->fblocks.size();
      int tpos[64];
      for (int& x : tpos) x = -1;
      for (int q = 0; q < dp.num_low; q++) tpos[q] = q;
      for (int i = 0; i < dp.num_high; i++) tpos[dp.hbits[i]] = dp.num_low + i;
      for (int bi : P.passes[pi].blocks) {
        FusedBlockDev db = P.dev_blocks[j++];
        auto local = [&](int q) {
          for (int c = 0; c < fused::kBlockQubits; c++)
            if (tpos[q] >= 0 && db.pos[c] == tpos[q]) return c;
          return -1;
        };
        FusedGenBlock gb{(uint32_t)h->gops.size(), 0};
        for (int oi : P.blocks[bi].ops) {
          const TapeOp& t = sub[oi];
          FusedGenOp g{};
          g.kind = (int8_t)t.kind;
          g.lt = (int8_t)local(t.q);
          g.lc = (int8_t)(t.ctrl >= 0 ? local(t.ctrl) : -1);
          g.p = t.p;
          if (g.lt < 0 || (t.ctrl >= 0 && g.lc < 0)) return false;
          h->gops.push_back(g);
          gb.num_ops++;
        }
        db.image = (uint32_t)h->fblocks.size();
        h->fblocks.push_back(db);
        h->gblocks.push_back(gb);
      }
      passes.push_back(dp);
    }
    h->fseg.push_back(std::move(passes));
  }
  return true;
}

int upload_programs(mlb_hea* h) {
  std::vector<AdjOp> all_ops;
  std::vector<int> all_slots;
  for (auto* vec : {&h->fwd, &h->bwd})
    for (auto& gp : *vec) {
      gp.ops_off = all_ops.size();
      gp.slots_off = all_slots.size();
      all_ops.insert(all_ops.end(), gp.ops.begin(), gp.ops.end());
      all_slots.insert(all_slots.end(), gp.param_of_slot.begin(), gp.param_of_slot.end());
    }
  std::vector<AdjTerm> all_terms;
  for (auto& tp : h->lam) {
    tp.terms_off = all_terms.size();
    all_terms.insert(all_terms.end(), tp.terms.begin(), tp.terms.end());
  }
  cudaError_t e = cudaMalloc((void**)&h->d_ops, std::max<size_t>(1, all_ops.size()) * sizeof(AdjOp));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_slots, std::max<size_t>(1, all_slots.size()) * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_terms, std::max<size_t>(1, all_terms.size()) * sizeof(AdjTerm));
  if (e != cudaSuccess) return cfail(e, "adjoint program upload");
  cudaMemcpy(h->d_ops, all_ops.data(), all_ops.size() * sizeof(AdjOp), cudaMemcpyHostToDevice);
  cudaMemcpy(h->d_slots, all_slots.data(), all_slots.size() * sizeof(int), cudaMemcpyHostToDevice);
  e = cudaMemcpy(h->d_terms, all_terms.data(), all_terms.size() * sizeof(AdjTerm), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cfail(e, "adjoint program upload");
  if (h->fused_ok) {
    e = cudaMalloc((void**)&h->d_fblocks, h->fblocks.size() * sizeof(FusedBlockDev));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_gblocks, h->gblocks.size() * sizeof(FusedGenBlock));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_gops, std::max<size_t>(1, h->gops.size()) * sizeof(FusedGenOp));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->d_ferr, sizeof(int));
    if (e != cudaSuccess) return cfail(e, "fused forward program upload");
    cudaMemcpy(h->d_fblocks, h->fblocks.data(), h->fblocks.size() * sizeof(FusedBlockDev), cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_gblocks, h->gblocks.data(), h->gblocks.size() * sizeof(FusedGenBlock), cudaMemcpyHostToDevice);
    e = cudaMemcpy(h->d_gops, h->gops.data(), h->gops.size() * sizeof(FusedGenOp), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cfail(e, "fused forward program upload");
  }
  return MLB_OK;
}

// Bits of the tile enumeration of a batch of B states of n qubits.
int batch_bits(uint32_t n, size_t B) {
  int b = 0;
  while (((size_t)1 << b) < B) b++;
  return (int)n + b;
}

// Whether this evaluation runs the forward sweep on the tensor cores
// (complex64 states only: the fused kernel works on FP32 amplitudes).
bool use_fused_forward(const mlb_hea* h, size_t B) {
  if (!h->fused_ok || h->fused_mode < 0 || h->dtype != MLB_C64) return false;
  return batch_bits(h->n, B) <= 13 + 24 && B <= 65535;  // the fused kernel's tile-index reach
}

int evaluate_chunk(mlb_hea* h, size_t B, const double* h_params, double* h_E, double* h_G, bool use_ckpt) {
  const size_t dim = (size_t)1 << h->n;
  const size_t ab = h->dtype == MLB_C128 ? 16 : 8;
  int rc;
  // 1. cos/sin table with host libm (gate_ry / gate_rz: cos(theta/2), sin(theta/2))
  std::vector<double2> cs(B * h->P);
  for (size_t i = 0; i < B * h->P; i++) cs[i] = make_double2(std::cos(h_params[i] / 2.0), std::sin(h_params[i] / 2.0));
  if ((rc = grow(h->d_cs, h->cs_cap, cs.size()))) return rc;
  cudaMemcpyAsync(h->d_cs, cs.data(), cs.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream);
  // buffers
  if (h->batch_cap < B) {
    if (h->psi) cudaFree(h->psi);
    if (h->lamb) cudaFree(h->lamb);
    h->psi = h->lamb = nullptr;
    h->batch_cap = 0;
    cudaError_t e = cudaMalloc(&h->psi, B * dim * ab);
    if (e == cudaSuccess) e = cudaMalloc(&h->lamb, B * dim * ab);
    if (e != cudaSuccess) return cfail(e, "psi/lambda allocation");
    h->batch_cap = B;
  }
  if (use_ckpt) {
    const size_t need = (h->fwd_seg.size() - 2) * B * dim * ab;
    if (h->ckpt_cap < need) {
      if (h->ckpt) cudaFree(h->ckpt);
      h->ckpt = nullptr;
      h->ckpt_cap = 0;
      cudaError_t e = cudaMalloc(&h->ckpt, need);
      if (e != cudaSuccess) return cfail(e, "checkpoint allocation");
      h->ckpt_cap = need;
    }
  }
  size_t max_slots_tiles = 1, max_tiles = 1;
  for (auto& gp : h->bwd) max_slots_tiles = std::max(max_slots_tiles, gp.P.tiles_per_state * B * (size_t)gp.P.num_slots);
  for (auto& tp : h->lam) max_tiles = std::max(max_tiles, tp.P.tiles_per_state * B);
  if ((rc = grow(h->d_part, h->part_cap, max_slots_tiles))) return rc;
  if ((rc = grow(h->d_epart, h->epart_cap, max_tiles))) return rc;
  if ((rc = grow(h->d_out, h->out_cap, B + B * h->P))) return rc;
  // 2. forward
  // |0...0>: the tape itself starts with X on the hf_reference bits (vqe.c:1953-1959)
  if ((rc = launch_adj_init(h->dtype, h->psi, (int)h->n, B, 0, h->stream))) return hfail(rc, "init kernel");
  const size_t nseg = h->fwd_seg.size() - 1;
  const size_t state_bytes = B * dim * ab;
  const bool fused = use_fused_forward(h, B);
  h->last_fused = fused ? 1 : 0;
  if (fused) {  // every vector's operand images, from the cos/sin table
    const size_t K = h->fblocks.size();
    if (h->images_cap < B * K * fused::kBImageBytes) {
      if (h->d_images) cudaFree(h->d_images);
      h->d_images = nullptr;
      h->images_cap = 0;
      cudaError_t e = cudaMalloc((void**)&h->d_images, B * K * fused::kBImageBytes);
      if (e != cudaSuccess) return cfail(e, "operand image allocation");
      h->images_cap = B * K * fused::kBImageBytes;
    }
    if ((rc = launch_fused_images(h->d_gblocks, (int)K, h->d_gops, h->d_cs, (int)h->P, (int)B, h->d_images,
                                  h->stream)))
      return hfail(rc, "operand image build");
    cudaMemsetAsync(h->d_ferr, 0, sizeof(int), h->stream);
  }
  for (size_t k = 0; k < nseg; k++) {
    if (fused) {
      for (FusedPassDev dp : h->fseg[k]) {
        dp.num_tiles = (uint64_t)B << (h->n - fused::kTileBits);
        dp.vec_shift = h->n - fused::kTileBits;
        dp.vec_images = (uint32_t)h->fblocks.size();
        if ((rc = launch_fused_pass(h->psi, batch_bits(h->n, B), dp, h->d_fblocks, h->d_images, h->d_ferr,
                                    h->num_sms, h->stream)))
          return hfail(rc, "fused forward pass");
      }
    } else {
      for (size_t i = h->fwd_seg[k]; i < h->fwd_seg[k + 1]; i++) {
        const GatePass& gp = h->fwd[i];
        AdjPass P = gp.P;
        P.num_tiles = P.tiles_per_state * B;
        if ((rc = launch_adj_gates(h->dtype, h->psi, nullptr, P, h->d_ops + gp.ops_off, h->d_cs, nullptr, false,
                                   false, h->num_sms, h->stream)))
          return hfail(rc, "forward pass");
      }
    }
    if (use_ckpt && k + 1 < nseg) {
      cudaError_t e = cudaMemcpyAsync((char*)h->ckpt + k * state_bytes, h->psi, state_bytes,
                                      cudaMemcpyDeviceToDevice, h->stream);
      if (e != cudaSuccess) return cfail(e, "checkpoint save");
    }
  }
  // The tensor-core forward shrinks |psi| slightly (its FP32 accumulation
  // rounds magnitudes down); energies and gradients both carry |psi|^2, so
  // they are divided by the forward state's squared norm at the end.
  if (fused) {
    if ((rc = grow(h->d_norm, h->norm_cap, B))) return rc;
    if ((rc = launch_batch_norm(h->psi, dim, B, h->d_norm, h->stream))) return hfail(rc, "forward norm");
  }
  // 3. lambda = H psi and the energies
  for (size_t k = 0; k < h->lam.size(); k++) {
    AdjPass P = h->lam[k].P;
    P.num_tiles = P.tiles_per_state * B;
    const bool last = k + 1 == h->lam.size();
    if ((rc = launch_adj_pauli(h->dtype, h->psi, h->lamb, P, h->d_terms + h->lam[k].terms_off, k > 0, last,
                               h->d_epart, h->num_sms, h->stream)))
      return hfail(rc, "lambda pass");
    if (last && (rc = launch_adj_reduce(h->d_epart, P.tiles_per_state, 1, B, nullptr, 1, h->d_out, h->stream)))
      return hfail(rc, "energy reduce");
  }
  // 4. backward
  if (h_G) {
    for (size_t j = 0; j < nseg; j++) {
      const size_t k = nseg - 1 - j;  // segment swept backwards
      if (use_ckpt && k + 1 < nseg) {  // psi at the end of segment k, as the forward sweep left it
        cudaError_t e = cudaMemcpyAsync(h->psi, (char*)h->ckpt + k * state_bytes, state_bytes,
                                        cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) return cfail(e, "checkpoint restore");
      }
    for (size_t i = h->bwd_seg[j]; i < h->bwd_seg[j + 1]; i++) {
      const GatePass& gp = h->bwd[i];
      AdjPass P = gp.P;
      P.num_tiles = P.tiles_per_state * B;
      if ((rc = launch_adj_gates(h->dtype, h->psi, h->lamb, P, h->d_ops + gp.ops_off, h->d_cs, h->d_part, true,
                                 true, h->num_sms, h->stream)))
        return hfail(rc, "backward pass");
      if (P.num_slots &&
          (rc = launch_adj_reduce(h->d_part, P.tiles_per_state, P.num_slots, B, h->d_slots + gp.slots_off,
                                  (int)h->P, h->d_out + B, h->stream)))
        return hfail(rc, "gradient reduce");
    }
    }
  }
  if (fused && (rc = launch_divide_by_norm(h->d_out, B, (int)h->P, h->d_norm, h->stream)))
    return hfail(rc, "norm correction");
  if (h_E) cudaMemcpyAsync(h_E, h->d_out, B * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (h_G) cudaMemcpyAsync(h_G, h->d_out + B, B * h->P * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  int ferr = 0;
  if (fused) cudaMemcpyAsync(&ferr, h->d_ferr, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cfail(e, "adjoint evaluation");
  if (ferr) return hfail(MLB_ERR_TIMEOUT, "fused forward pass: tensor-core completion wait ran out");
  return MLB_OK;
}

// The quantum geometric tensor of the ansatz at one parameter vector.
// A rotation R(t) = exp(-i t G / 2) (G = Y for RY, Z for RZ) satisfies
// G R(t) = i R(t + pi), so the reference's derivative state
// d_i psi = (-i/2) U_after G_i U_upto |hf> (vqe_qng.c:60-99) equals
// (1/2) psi(theta + pi e_i): the ansatz with parameter i's cos/sin pair
// (c, s) replaced by (-s, c), exactly.  psi and the P shifted states run as
// one batch of P + 1 vectors through the forward passes, and the Gram
// matrix of the batch gives every inner product:
//   <psi|d_i psi> = G[0][i+1] / 2,  <d_i psi|d_j psi> = G[i+1][j+1] / 4.
// Q_ij = <d_i psi|d_j psi> - conj(<psi|d_i psi>) <psi|d_j psi>; the metric
// and the curvature are filled as vqe_compute_qgt (vqe_qng.c:166-196) and
// vqe_compute_berry_curvature (:198-232) fill them.
int geometry(mlb_hea* h, const double* params, double* metric, double* curvature) {
  if (h->dtype != MLB_C128) return hfail(MLB_ERR_NOT_SUPPORTED, "geometry needs a complex128 problem");
  const size_t P = h->P, B = P + 1;
  const size_t dim = (size_t)1 << h->n;
  int rc;
  std::vector<double2> cs(B * P);
  for (size_t p = 0; p < P; p++) cs[p] = make_double2(std::cos(params[p] / 2.0), std::sin(params[p] / 2.0));
  for (size_t i = 0; i < P; i++) {
    std::memcpy(&cs[(i + 1) * P], cs.data(), P * sizeof(double2));
    cs[(i + 1) * P + i] = make_double2(-cs[i].y, cs[i].x);
  }
  if ((rc = grow(h->d_cs, h->cs_cap, cs.size()))) return rc;
  cudaMemcpyAsync(h->d_cs, cs.data(), cs.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream);
  if (h->batch_cap < B) {
    if (h->psi) cudaFree(h->psi);
    if (h->lamb) cudaFree(h->lamb);
    h->psi = h->lamb = nullptr;
    h->batch_cap = 0;
    cudaError_t e = cudaMalloc(&h->psi, B * dim * 16);
    if (e == cudaSuccess) e = cudaMalloc(&h->lamb, B * dim * 16);
    if (e != cudaSuccess) return cfail(e, "geometry: P + 1 states");
    h->batch_cap = B;
  }
  const size_t gbytes = B * B * sizeof(double2);
  const size_t need = gbytes + gram_scratch_bytes((int)B, dim, h->num_sms);
  size_t cap = h->gram_cap;
  if ((rc = grow(h->d_gram, cap, (need + 255) / 256 * 256))) return rc;
  h->gram_cap = cap;
  if ((rc = launch_adj_init(h->dtype, h->psi, (int)h->n, B, 0, h->stream))) return hfail(rc, "init kernel");
  for (const GatePass& gp : h->fwd) {
    AdjPass Pp = gp.P;
    Pp.num_tiles = Pp.tiles_per_state * B;
    if ((rc = launch_adj_gates(h->dtype, h->psi, nullptr, Pp, h->d_ops + gp.ops_off, h->d_cs, nullptr, false,
                               false, h->num_sms, h->stream)))
      return hfail(rc, "forward pass");
  }
  double2* d_G = reinterpret_cast<double2*>(h->d_gram);
  if ((rc = launch_gram(h->psi, dim, (int)B, d_G, h->d_gram + (gbytes + 255) / 256 * 256, h->num_sms, h->stream)))
    return hfail(rc, "Gram kernel");
  std::vector<double2> G(B * B);
  cudaMemcpyAsync(G.data(), d_G, gbytes, cudaMemcpyDeviceToHost, h->stream);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cfail(e, "geometry");
  // a register padded to 3 qubits (n < 3) carries the idle qubits in |0>:
  // the inner products are those of the n-qubit problem
  std::vector<double> ovr(P), ovi(P);
  for (size_t i = 0; i < P; i++) {
    ovr[i] = G[i + 1].x * 0.5;  // row 0: <psi|psi_{i+1}>
    ovi[i] = G[i + 1].y * 0.5;
  }
  for (size_t i = 0; i < P; i++)
    for (size_t j = i; j < P; j++) {
      const double2 g = G[(i + 1) * B + (j + 1)];
      const double ar = g.x * 0.25, ai = g.y * 0.25;
      // conj(ov_i) * ov_j
      const double cr = ovr[i] * ovr[j] + ovi[i] * ovi[j];
      const double ci = ovr[i] * ovi[j] - ovi[i] * ovr[j];
      if (metric) {
        const double v = ar - cr;
        metric[i * P + j] = v;
        metric[j * P + i] = v;
      }
      if (curvature) {
        if (i == j) {
          curvature[i * P + i] = 0.0;
        } else {
          const double F = -2.0 * (ai - ci);
          curvature[i * P + j] = F;
          curvature[j * P + i] = -F;
        }
      }
    }
  return MLB_OK;
}

}  // namespace

extern "C" {

int mlb_hea_geometry(mlb_hea_t* h, const double* params, double* metric, double* curvature) {
  if (!h || !params) return hfail(MLB_ERR_INVALID_ARG, "null argument");
  Guard g(h->device);
  return geometry(h, params, metric, curvature);
}

int mlb_hea_create(uint32_t n, uint32_t layers, uint64_t hf, size_t num_terms, const uint64_t* xm,
                   const uint64_t* zm, const double* coeffs, int dtype, int device, mlb_hea_t** out) {
  if (!out) return hfail(MLB_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  if (n < 1 || n > 30 || layers < 1) return hfail(MLB_ERR_NUM_QUBITS, "need 1 <= N <= 30 and L >= 1");
  if (dtype != MLB_C128 && dtype != MLB_C64) return hfail(MLB_ERR_INVALID_ARG, "dtype");
  if (num_terms && (!xm || !zm || !coeffs)) return hfail(MLB_ERR_INVALID_ARG, "null term arrays");
  const uint64_t allm = (1ull << n) - 1ull;
  if (hf & ~allm) return hfail(MLB_ERR_INVALID_QUBIT, "hf_reference outside the register");
  for (size_t t = 0; t < num_terms; t++)
    if ((xm[t] | zm[t]) & ~allm) return hfail(MLB_ERR_INVALID_QUBIT, "Pauli term %zu outside the register", t);
  int cnt = 0;
  if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
    cudaGetLastError();
    return hfail(MLB_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= cnt) return hfail(MLB_ERR_NO_DEVICE, "device %d", device);
  Guard g(device);
  auto* h = new mlb_hea();
  // Registers below 3 qubits run padded with idle qubits (kept in |0>): the
  // passes' register groups span 3 qubits.  Energies and gradients are those
  // of the n-qubit problem.
  h->n = n < 3 ? 3 : n;
  h->layers = layers;
  h->P = 2 * n * layers;
  h->hf = hf;
  h->dtype = dtype;
  h->device = device;
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
  h->xm.assign(xm, xm + num_terms);
  h->zm.assign(zm, zm + num_terms);
  h->coeff.assign(coeffs, coeffs + num_terms);
  if (num_terms == 0) {  // H = 0: keep one zero term so lambda is defined
    h->xm.push_back(0);
    h->zm.push_back(0);
    h->coeff.push_back(0.0);
  }
  for (uint32_t q = 0; q < n; q++)
    if (hf >> q & 1ull) h->tape.push_back({ADJ_KIND_X, (int)q, -1, -1});
  int p = 0;
  for (uint32_t l = 0; l < layers; l++) {
    for (uint32_t q = 0; q < n; q++) {
      h->tape.push_back({ADJ_KIND_RY, (int)q, -1, p++});
      h->tape.push_back({ADJ_KIND_RZ, (int)q, -1, p++});
    }
    for (uint32_t q = 0; q + 1 < n; q++) h->tape.push_back({ADJ_KIND_X, (int)q + 1, (int)q, -1});
  }
  // segments of s = ceil(sqrt(L)) layers (the hf X prefix joins segment 0)
  h->seg_layers = (uint32_t)std::ceil(std::sqrt((double)layers));
  const size_t per_layer = 3 * (size_t)n - 1, prefix = h->tape.size() - per_layer * layers;
  std::vector<size_t> cut{0};
  for (uint32_t l = h->seg_layers; l < layers; l += h->seg_layers) cut.push_back(prefix + l * per_layer);
  cut.push_back(h->tape.size());
  h->fwd_seg.push_back(0);
  for (size_t k = 0; k + 1 < cut.size(); k++) {
    std::vector<TapeOp> sub(h->tape.begin() + cut[k], h->tape.begin() + cut[k + 1]);
    plan_gates(h, sub, false, h->fwd);
    h->fwd_seg.push_back(h->fwd.size());
  }
  h->bwd_seg.push_back(0);
  for (size_t k = cut.size() - 1; k-- > 0;) {
    std::vector<TapeOp> rev(h->tape.rend() - cut[k + 1], h->tape.rend() - cut[k]);
    plan_gates(h, rev, true, h->bwd);
    h->bwd_seg.push_back(h->bwd.size());
  }
  plan_terms(h);
  // the tensor-core forward sweep's plans (used by complex64 problems by default)
  if (dtype == MLB_C64 && h->n == n && n >= (uint32_t)fused::kTileBits) {
    h->fused_ok = plan_fused_forward(h, cut);
    if (!h->fused_ok) {
      h->fseg.clear();
      h->fblocks.clear();
      h->gblocks.clear();
      h->gops.clear();
    }
  }
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return hfail(MLB_ERR_DRIVER, "stream creation");
  }
  int rc = upload_programs(h);
  if (rc) {
    mlb_hea_free(h);
    return rc;
  }
  *out = h;
  return MLB_OK;
}

void mlb_hea_free(mlb_hea_t* h) {
  if (!h) return;
  Guard g(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (void* p : {h->psi, h->lamb, h->ckpt, (void*)h->d_cs, (void*)h->d_part, (void*)h->d_epart,
                  (void*)h->d_ops, (void*)h->d_terms, (void*)h->d_slots, (void*)h->d_out, (void*)h->d_gram,
                  (void*)h->d_fblocks, (void*)h->d_gblocks, (void*)h->d_gops, (void*)h->d_images,
                  (void*)h->d_ferr, (void*)h->d_norm})
    if (p) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int mlb_hea_num_parameters(const mlb_hea_t* h, uint32_t* out) {
  if (!h || !out) return hfail(MLB_ERR_INVALID_ARG, "null argument");
  *out = h->P;
  return MLB_OK;
}

int mlb_hea_set_memory_budget(mlb_hea_t* h, size_t bytes) {
  if (!h) return hfail(MLB_ERR_INVALID_ARG, "null problem");
  h->budget = bytes;
  return MLB_OK;
}

int mlb_hea_plan_stats(const mlb_hea_t* h, uint32_t* fwd_passes, uint32_t* lam_passes, uint32_t* bwd_passes) {
  if (!h) return hfail(MLB_ERR_INVALID_ARG, "null problem");
  if (fwd_passes) *fwd_passes = (uint32_t)h->fwd.size();
  if (lam_passes) *lam_passes = (uint32_t)h->lam.size();
  if (bwd_passes) *bwd_passes = (uint32_t)h->bwd.size();
  return MLB_OK;
}

int mlb_hea_evaluate(mlb_hea_t* h, size_t batch, const double* params, double* energies, double* grads,
                     int on_device) {
  if (!h || !params) return hfail(MLB_ERR_INVALID_ARG, "null argument");
  if (batch == 0) return MLB_OK;
  Guard g(h->device);
  const size_t P = h->P;
  // host copies when the caller passes device pointers
  std::vector<double> hp, hE, hG;
  const double* p_in = params;
  if (on_device) {
    hp.resize(batch * P);
    cudaError_t e = cudaMemcpy(hp.data(), params, batch * P * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cfail(e, "parameter readback");
    p_in = hp.data();
  }
  if (energies) hE.resize(batch);
  if (grads) hG.resize(batch * P);
  // sub-batches within the memory budget
  const size_t sb = ((size_t)1 << h->n) * (h->dtype == MLB_C128 ? 16 : 8);  // one state
  const size_t extra = h->fwd_seg.size() - 2;                                  // checkpoints per vector
  size_t budget = h->budget;
  if (!budget) {  // 80 % of what is free, counting buffers this problem already holds
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    budget = (size_t)((fr + h->batch_cap * 2 * sb + h->ckpt_cap) * 0.8);
  }
  // checkpoints when they fit with the whole batch (mode 1: always; -1: never)
  bool use_ckpt = extra > 0 && grads != nullptr && h->ckpt_mode >= 0 &&
                  (h->ckpt_mode == 1 || budget / ((2 + extra) * sb) >= batch);
  const size_t img = use_fused_forward(h, batch) ? h->fblocks.size() * fused::kBImageBytes : 0;  // per vector
  const size_t per = (2 + (use_ckpt ? extra : 0)) * sb + img;
  size_t chunk = std::max<size_t>(1, budget / per);
  chunk = std::min(chunk, batch);
  h->last_ckpt = use_ckpt ? 1 : 0;
  h->last_chunks = (batch + chunk - 1) / chunk;
  for (size_t b0 = 0; b0 < batch; b0 += chunk) {
    const size_t nb = std::min(chunk, batch - b0);
    int rc = evaluate_chunk(h, nb, p_in + b0 * P, energies ? hE.data() + b0 : nullptr,
                            grads ? hG.data() + b0 * P : nullptr, use_ckpt);
    if (rc) return rc;
  }
  if (energies) {
    if (on_device) cudaMemcpy(energies, hE.data(), batch * sizeof(double), cudaMemcpyHostToDevice);
    else std::memcpy(energies, hE.data(), batch * sizeof(double));
  }
  if (grads) {
    if (on_device) cudaMemcpy(grads, hG.data(), batch * P * sizeof(double), cudaMemcpyHostToDevice);
    else std::memcpy(grads, hG.data(), batch * P * sizeof(double));
  }
  return MLB_OK;
}

int mlb_hea_set_fused_forward(mlb_hea_t* h, int mode) {
  if (!h) return hfail(MLB_ERR_INVALID_ARG, "null problem");
  if (mode < -1 || mode > 1) return hfail(MLB_ERR_INVALID_ARG, "mode must be -1, 0 or 1");
  if (mode == 1 && !h->fused_ok)
    return hfail(MLB_ERR_NOT_SUPPORTED, "no fused forward plan (complex64 and N >= 13 only)");
  h->fused_mode = mode;
  return MLB_OK;
}

int mlb_hea_last_forward_fused(const mlb_hea_t* h, int* fused, uint32_t* passes, uint32_t* blocks) {
  if (!h) return hfail(MLB_ERR_INVALID_ARG, "null problem");
  if (fused) *fused = h->last_fused;
  size_t np = 0;
  for (const auto& seg : h->fseg) np += seg.size();
  if (passes) *passes = (uint32_t)np;
  if (blocks) *blocks = (uint32_t)h->fblocks.size();
  return MLB_OK;
}

int mlb_hea_set_checkpointing(mlb_hea_t* h, int mode) {
  if (!h) return hfail(MLB_ERR_INVALID_ARG, "null problem");
  if (mode < -1 || mode > 1) return hfail(MLB_ERR_INVALID_ARG, "mode must be -1, 0 or 1");
  h->ckpt_mode = mode;
  return MLB_OK;
}

int mlb_hea_last_eval_stats(const mlb_hea_t* h, uint32_t* segment_layers, int* checkpoints_used,
                            size_t* sub_batches) {
  if (!h) return hfail(MLB_ERR_INVALID_ARG, "null problem");
  if (segment_layers) *segment_layers = h->seg_layers;
  if (checkpoints_used) *checkpoints_used = h->last_ckpt;
  if (sub_batches) *sub_batches = h->last_chunks;
  return MLB_OK;
}

const char* mlb_hea_last_error(void) { return g_herr.c_str(); }

}  // extern "C"
