// mlb_internal.h -- internal types shared by the engine's CUDA kernels and its
// host runtime.  Not part of the C ABI (include/moonlab_b200.h is).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "moonlab_b200.h"

namespace mlb {

// ---------------------------------------------------------------------------
// Device-side op encoding.  The host planner lowers mlb_op_t into these
// "local" ops for one tile pass: qubit positions are rewritten into the
// tile's local index space (bits 0..L-1 = global bits 0..L-1, bit L+k =
// global bit high[k]); controls and diagonal qubits outside the tile become
// per-tile predicates evaluated on the tile's base index.
// ---------------------------------------------------------------------------
enum DevOpKind : int32_t {
  DOP_1Q_GEN = 0,    // generic 2x2 on register bit rt
  DOP_1Q_REAL = 1,   // real 2x2 (RY-like)
  DOP_X = 2,         // swap pair
  DOP_DIAG1 = 3,     // diag(d0, d1) keyed on local bit lt (or outside bit)
  DOP_PHASE = 4,     // multiply by d0 where (loc & lmask)==lmask (outside part via omask)
  DOP_ZZ = 5,        // d0 if parity even else d1 over local mask lmask ^ outside parity
  DOP_2Q_GEN = 6,    // 4x4 on register bits (rt = low, rt2 = high)
  DOP_SWAP = 7,      // swap bits rt <-> rt2
  DOP_DENSE = 8,     // dense 2^k block (fused c64); matrix in the pass matrix pool
};

struct DevOp {
  int32_t kind;
  int32_t rt;        // register-group bit of the (low) target
  int32_t rt2;       // second register-group bit (2Q / SWAP)
  int32_t lt;        // local bit of the diagonal key (-1: outside the tile)
  uint32_t lcmask;   // local control mask (tile-local bits)
  uint32_t lmask;    // local mask (PHASE / ZZ)
  uint64_t ocmask;   // outside control mask (global bits); op skipped unless all set
  uint64_t omask;    // outside diagonal mask (global bits): ZZ parity / DIAG1 key / PHASE
  int32_t k;         // DENSE: number of qubits; 2Q (shared-memory segment): local bit of target2
  int32_t mat_off;   // DENSE: offset (in complex entries) into the matrix pool
  double m[32];      // matrix payload (same layout as mlb_op_t.m)
};

// One segment = consecutive ops whose non-diagonal targets fit in R
// register bits; each thread loads a 2^R-amplitude group into registers.
struct DevSegment {
  int32_t op_begin, op_end;
  int32_t nbits;        // number of active register bits (<= R)
  int32_t bits[4];      // local bit positions of the register bits (ascending)
  int32_t mode;         // 0: register groups; 1: one generic 4x4 op applied in shared memory;
                        // 2: dense 16x16 matrix (complex128) of the ops [op_begin, op_end)
  int32_t dense;        // mode 2: index into the program's dense segments
};

constexpr int kMaxHigh = 16;
// complex128 tile passes: tiles of 2^12 amplitudes (64 KiB, two CTAs per SM)
// with 2 contiguous low qubits (64-byte rows) and 10 chosen high ones
constexpr int kTileBitsC128 = 12;
constexpr int kLowBitsC128 = 2;  // contiguous low qubits of a complex128 tile (planner.h)
// A pass's op program is decoded into shared memory; the planner keeps every
// pass within these sizes.
constexpr int kMaxPassOps = 160;
constexpr int kMaxPassSegs = 160;

struct DevPass {
  int32_t n;            // qubits of the state
  int32_t L;            // low contiguous local bits
  int32_t H;            // high local bits
  int32_t num_segments;
  int32_t high[kMaxHigh];
  uint64_t num_tiles;   // 2^(n - L - H)
  uint64_t tile_free_mask; // global bits that enumerate tiles (not in the tile)
};

// ---- dense complex128 segments (dense.h, kernels_tile.cu) ----
// A register segment of a complex128 tile pass applied as one 16x16 complex
// matrix on its 4 register qubits, on the FP64 tensor cores (mma.sync m8n8k4
// f64) as three real 16x16 products (Gauss: Re U . Re x, Im U . Im x and
// (Re U + Im U) . (Re x + Im x)).  The matrix may depend on up to
// kDenseMaxCond conditioning qubits
// outside the register set (controls or diagonal keys; tile-local ones vary
// by group, outside ones by tile): one matrix variant per value of those
// bits.  Offsets are in 16-byte tile elements, already swizzled (the tile
// swizzle is linear over GF(2)).
constexpr int kDenseGroupBits = kTileBitsC128 - 4;   // 256 groups of 16 amplitudes per tile
constexpr int kDenseColBits = kDenseGroupBits - 3;   // 32 column tiles of 8 groups
constexpr int kDenseMaxCond = 6;     // conditioning qubits in all (64 variants)
constexpr int kDenseMaxCondLoc = kDenseColBits - 1;  // of them tile-local (the top group-index bits; a column-tile pair shares one)
constexpr int kDenseMaxCondOut = 6;  // of them outside the tile
// doubles per matrix variant: Re U and Im U as 2 x 8 A fragments of 32 lanes
constexpr int kDenseVarDoubles = 512;
struct DenseSegDev {
  uint32_t frag_off;   // first double of variant 0 in the fragment pool (kDenseVarDoubles per variant)
  uint8_t nloc;        // tile-local conditioning qubits: the top nloc group-index bits
  uint8_t nout;        // outside conditioning qubits: global bits obit[0 .. nout)
  uint8_t pad[2];
  uint8_t obit[8];
  uint16_t amp_off[16];  // fragment slot a -> offset
  uint16_t g_lo[8];      // group-index bits 0..2 -> offset
  uint16_t g_hi[1 << kDenseColBits];  // group-index bits 3.. -> offset
};
// Swizzle of a complex128 tile in shared memory (16-byte elements, 8 per
// 128-byte row): bits 0..2 (the bank group) xor the fold of all higher bits
// in 3-bit chunks, so every tile bit p moves the bank group (by bit p mod 3).
// Linear over GF(2) and a bijection (bits >= 3 are unchanged).
__host__ __device__ inline uint32_t tile_swz16(uint32_t e) {
  return e ^ (((e >> 3) ^ (e >> 6) ^ (e >> 9) ^ (e >> 12)) & 7u);
}

// ---------------------------------------------------------------------------
// Adjoint-gradient passes (kernels_adjoint.cu).  A pass covers a batch of
// states stored back to back, [B][2^n]; tiles never span two states.
// ---------------------------------------------------------------------------
constexpr int kMaxAdjOps = 160;
constexpr int kMaxAdjSegs = 64;
constexpr int kMaxAdjSlots = 96;   // parameter gradients accumulated per pass
constexpr int kMaxAdjTerms = 128;  // Pauli terms per lambda pass
enum AdjKind : int32_t { ADJ_KIND_X = 0, ADJ_KIND_RY = 1, ADJ_KIND_RZ = 2 };

struct AdjOp {
  int32_t kind;      // ADJ_KIND_*; X with a control mask is CNOT
  int32_t rt;        // register bit of the target (X, RY)
  int32_t lt;        // RZ: local bit of the target, -1 when outside the tile
  int32_t qt;        // RZ: global target qubit (tile-constant key when outside)
  int32_t p;         // parameter index (RY, RZ), -1 otherwise
  int32_t slot;      // backward: gradient slot of this pass, -1 none
  uint32_t lcmask;   // local control mask (CNOT control inside the tile)
  uint32_t pad;
  uint64_t ocmask;   // outside control mask (global bits)
};
struct AdjSeg {
  int32_t op_begin, op_end;
  int32_t bits[3];   // register bits (ascending local bit positions)
};
struct AdjTerm {     // one Pauli string restricted to a tile
  uint32_t xl, zl;   // local X / Z masks
  uint64_t zo;       // Z mask outside the tile (global bits)
  double cr, ci;     // c_k * i^{#Y}
};
struct AdjPass {
  int32_t n, L, H;
  int32_t num_ops, num_segments, num_slots, num_params;
  int32_t high[kMaxHigh];
  uint64_t tiles_per_state, num_tiles, tile_free_mask;
  AdjSeg segs[kMaxAdjSegs];
};
int adj_tile_bits(int dtype, bool dual);
int launch_adj_init(int dtype, void* psi, int n, uint64_t batch, uint64_t hf, cudaStream_t stream);
int launch_adj_gates(int dtype, void* psi, void* lam, const AdjPass& P, const AdjOp* d_ops, const double2* d_cs,
                     double* d_partials, bool dual, bool backward, int num_sms, cudaStream_t stream);
int launch_adj_pauli(int dtype, const void* psi, void* lam, const AdjPass& P, const AdjTerm* d_terms,
                     bool accumulate, bool energy, double* d_epart, int num_sms, cudaStream_t stream);
int launch_adj_reduce(const double* d_partials, uint64_t tiles_per_state, int num_slots, uint64_t batch,
                      const int* d_param_of_slot, int num_params, double* d_out, cudaStream_t stream);
// d_norm[b] = |psi_b|^2 of a complex64 batch; then d_out ([B] energies,
// [B][P] gradients) divided by it.
int launch_batch_norm(const void* psi_c64, uint64_t dim, uint64_t batch, double* d_norm, cudaStream_t stream);
int launch_divide_by_norm(double* d_out, uint64_t batch, int num_params, const double* d_norm,
                          cudaStream_t stream);

// Gram matrix of B complex128 states stored back to back ([B][dim]):
// d_G[a * B + b] = sum_x conj(S_a[x]) S_b[x] for a <= b (the rest of d_G is
// not written), in FP64 with a fixed summation order (kernels_geometry.cu).
// d_scratch: gram_scratch_bytes(B, dim, num_sms) bytes of device memory.
size_t gram_scratch_bytes(int B, uint64_t dim, int num_sms);
int launch_gram(const void* states, uint64_t dim, int B, double2* d_G, void* d_scratch, int num_sms,
                cudaStream_t stream);

// Kernel launchers (kernels_*.cu).  All asynchronous on `stream`.
// d_dsegs / d_frags: the program's dense segments and their matrix fragments
// (complex128 segments of mode 2; may be null when there are none).
// all_dense: every segment of the pass is a dense complex128 segment (mode
// 2); such passes run a kernel that holds only the dense code.
int launch_tile_pass(int dtype, void* amp, const DevPass& pass, const DevSegment* d_segs,
                     const DevOp* d_ops, const DenseSegDev* d_dsegs, const double* d_frags, int num_sms,
                     cudaStream_t stream, bool all_dense = false);
// Sets the tile kernel's function attributes on the current device (done
// lazily by launch_tile_pass; called before a stream capture).
void prepare_tile_launch(int dtype);
// The current device's FP64 tensor-core throughput (mma.sync m8n8k4 f64,
// register operands), best of three timed launches after a warm-up.
int measure_fp64_tensor_peak(int num_sms, double* tflops);
int launch_gate(int dtype, void* amp, int n, const mlb_op_t& op, cudaStream_t stream);
int launch_init_zero(int dtype, void* amp, int n, cudaStream_t stream);
int launch_convert(int dst_dtype, void* dst, int src_dtype, const void* src, uint64_t dim,
                   cudaStream_t stream);

// Reductions: results written into a device FP64 scratch block, then copied.
int launch_reduce_probs_z(int dtype, const void* amp, int n, double* d_out /* n+1 */,
                          double* d_partials, int num_sms, cudaStream_t stream);
// Pauli strings sharing one X mask (<= 16 per call); out_terms[t] = Re<P_t>.
int launch_pauli_group(int dtype, const void* amp, int n, uint64_t xmask, int num_terms,
                       const uint64_t* d_zmasks, const int* d_nys, double* d_out_terms,
                       double* d_partials, int num_sms, cudaStream_t stream);
int launch_probabilities(int dtype, const void* amp, int n, int rule, double* d_out,
                         cudaStream_t stream);
int launch_scale(int dtype, void* amp, int n, double factor, uint64_t zero_mask,
                 uint64_t zero_val, cudaStream_t stream);

// Exact reproduction of the reference's sequential FP64 sums
// (kernels_sample.cu).  Both synchronize `stream` before returning.
int sample_exact(int dtype, const void* amp, int n, int rule, const double* h_uniforms,
                 size_t num, uint64_t* h_out, int num_sms, cudaStream_t stream,
                 char* errbuf, size_t errlen);
// Left-to-right sum over indices with (i & fmask) == fval of cabs(a_i)^2:
// fused = false: s = fl(s + fl(h*h)); fused = true: s = fma(h, h, s).
int seq_sum_exact(int dtype, const void* amp, int n, uint64_t fmask, uint64_t fval, bool fused,
                  int num_sms, cudaStream_t stream, double* total);

uint64_t kernel_launch_count();
void count_launch(uint64_t k = 1);

// Records the message mlb_last_error() returns on this thread; returns code.
int record_error(int code, const char* msg);

// ---- fused complex64 path (kernels_fused.cu, planned by fused.h) ----------
// A dense 5-qubit block inside a 13-qubit tile: pos = its tile bit positions
// (block index bit j <-> tile bit pos[j]), q = the other 8 tile positions in
// increasing order (row index bit i <-> tile bit q[i]), image = index of its
// 16 KiB operand image (bf16 hi then lo, K-major 128-byte swizzle).
struct FusedBlockDev {
  uint8_t pos[5];
  uint8_t q[8];
  uint8_t pad[3];
  uint32_t image;
};
// A fused pass: tile = qubits 0..num_low-1 (tile bits 0..num_low-1) plus
// hbits[0..num_high-1] (tile bits num_low + i), num_low + num_high = 13;
// blocks [block_begin, block_begin + num_blocks) applied in order to every
// tile.
struct FusedPassDev {
  uint8_t hbits[12];
  uint8_t num_low;
  uint8_t num_high;
  uint8_t pad[2];
  uint64_t num_tiles;
  uint32_t block_begin;
  uint32_t num_blocks;
  // per-vector operand images (a batch of states with their own matrices):
  // tile t uses image (block image + (t >> vec_shift) * vec_images);
  // vec_shift = 63 when every tile shares one set
  uint32_t vec_shift;
  uint32_t vec_images;
  // bit 63 set: the tile index is deposited into the other set bits of
  // free_mask (the pass runs over only those tiles); else into every bit
  // outside the tile
  uint64_t free_mask;
};
// ---- small circuits in one launch (kernels_small.cu; the serving path) ----
// One request per item: ops[ops_off .. ops_off + num_ops) on an n-qubit
// state from |0...0>, then shots outcomes for uniforms[uni_off ..] written
// to outcomes[out_off ..].
struct SmallItem {
  uint64_t ops_off, uni_off, out_off;
  uint32_t num_ops, n, shots, pad;
};
int small_max_qubits(int dtype);  // 12 (complex128) / 13 (complex64): the state fits a CTA
int launch_small_circuits(int dtype, const SmallItem* d_items, int num_items, const mlb_op_t* d_ops,
                          const double* d_uniforms, unsigned long long* d_outcomes, uint32_t nmax,
                          int num_sms, cudaStream_t stream);
// Gate records -> validated, canonical ops with 1q runs fused (what a flush
// of mlb_run_gates would plan).
int prepare_ops(const mlb_gate_t* gates, size_t num_gates, uint32_t n, std::vector<mlb_op_t>& out);

// ---- persistent small-circuit loop (kernels_mailbox.cu; mailbox.cpp) ----
struct MailboxItem {  // one request, in ring slot seq % slots
  uint32_t num_ops, n, shots, pad;
};
struct MailboxDev {
  const MailboxItem* items;        // [slots]
  const mlb_op_t* ops;             // [slots][max_ops]
  const double* uniforms;          // [slots][max_shots]
  unsigned long long* outcomes;    // mapped host memory, [slots][max_shots]
  uint64_t* done;                  // mapped host memory, [slots]: seq + 1 once slot's request is done
  uint64_t* head;                  // next sequence number to claim
  const uint64_t* tail;            // requests published so far
  const uint32_t* stop;            // non-zero: blocks exit
  uint32_t* exited;                // blocks that have left this launch
  int* end_status;                 // MLB_OK (stopped) or MLB_ERR_TIMEOUT (idle limit), by the last block
  uint64_t idle_ns;
  uint32_t slots, max_ops, max_shots, nmax;
};
size_t mailbox_smem_bytes(int dtype);
int launch_mailbox(int dtype, const MailboxDev& mb, int ctas, cudaStream_t stream);

// ---- per-vector operand images of fused blocks (kernels_fused.cu) ----
// A block's gates in the block's own 5 qubits (the local bit of a qubit is
// the index of its tile position among the block's sorted positions), for
// parameterised circuits whose angles differ per batch vector.
struct FusedGenOp {
  int8_t kind;  // ADJ_KIND_X (a CNOT when lc >= 0), ADJ_KIND_RY, ADJ_KIND_RZ
  int8_t lt;    // local target bit
  int8_t lc;    // local control bit, -1: none
  int8_t pad;
  int32_t p;    // parameter (RY, RZ): cs[vector * num_params + p] = (cos, sin) of half the angle
};
struct FusedGenBlock {
  uint32_t op_begin, num_ops;
};
// images[(v * num_blocks + k) * 16 KiB]: block k's operand image for vector v,
// the layout the fused host planner writes (bf16 hi and lo of
// [Re U -Im U; Im U Re U], K-major, 128-byte swizzle).
int launch_fused_images(const FusedGenBlock* blocks, int num_blocks, const FusedGenOp* ops, const double2* cs,
                        int num_params, int batch, uint8_t* images, cudaStream_t stream);

// d_err: device word set non-zero if a tensor-core completion wait ran out.
int launch_fused_pass(void* amp, int n, const FusedPassDev& pass, const FusedBlockDev* d_blocks,
                      const uint8_t* d_images, int* d_err, int num_sms, cudaStream_t stream, int test_skip_copy = 0);

}  // namespace mlb
