// engine.cpp -- host runtime of the B200 state-vector engine and its C ABI
// (include/moonlab_b200.h).
//
// A state owns its HBM buffer, a CUDA stream and a host-side queue of gate
// ops.  Gate calls only validate, canonicalise and queue; the queue is
// flushed at the next read, synchronize or explicit flush.  A flush lowers
// the queue into tile passes (kernels_tile.cu): the planner greedily picks
// the high qubits of each pass so that as many queued ops as possible run
// in one read+write of the state, keeping program order between ops that
// share a qubit.  Controls and diagonal qubits never need to be inside a
// tile (they are constant over it), so CNOT ladders and ZZ layers cost no
// tile room for their controls / phases.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dense.h"
#include "fused.h"
#include "mlb_internal.h"
#include "planner.h"

extern "C" {
void mlb_mat_rx(double theta, double m[8]);
void mlb_mat_ry(double theta, double m[8]);
void mlb_mat_rz(double theta, double m[8]);
void mlb_mat_phase1(int which, double theta, double m[8]);
void mlb_mat_zz(double theta, double out[4]);
void mlb_mat_cphase(double theta, double out[2]);
void mlb_mat_crz_inner(double theta, double m[8]);
}

namespace mlb {
static std::atomic<uint64_t> g_launches{0};
uint64_t kernel_launch_count() { return g_launches.load(); }
void count_launch(uint64_t k) { g_launches.fetch_add(k); }
}  // namespace mlb

using namespace mlb;
using namespace mlb::plan;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? MLB_ERR_OUT_OF_MEMORY : MLB_ERR_DRIVER, "%s: %s", what,
              cudaGetErrorString(e));
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

int mlb::record_error(int code, const char* msg) { return fail(code, "%s", msg); }

struct mlb_state {
  uint32_t n = 0;
  int dtype = MLB_C128;
  int device = 0;
  void* amp = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  int mode = MLB_EXEC_TILED;
  bool fuse1q = true;
  bool dense_c128 = true;  // complex128 register segments as dense matrices on the FP64 tensor cores
  int num_sms = 148;
  std::vector<mlb_op_t> queue;
  // device scratch for reductions
  double* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  // plan upload buffers
  void* d_plan = nullptr;
  size_t d_plan_bytes = 0;
  void* h_plan = nullptr;
  size_t h_plan_bytes = 0;
  cudaEvent_t plan_ev = nullptr;
  bool plan_ev_pending = false;
  bool timing = false;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  bool timed_pending = false;
  mlb_flush_stats_t stats{};
  // fused path: device error word of the tensor-core kernel and its host copy
  int* d_ferr = nullptr;
  int* h_ferr = nullptr;
  bool ferr_pending = false;
  bool test_skip_copy = false;  // mlb_test_fused_skip_copy: the next fused flush only
  // Qubits that may be 1 in the index of a nonzero amplitude: every
  // amplitude whose index has a bit outside `support` is exactly 0.  A reset
  // makes it 0.  A tile pass mixes amplitudes only within its tiles, so it
  // runs over the tiles whose outside bits lie in `support` (the others are
  // zero and stay zero) and then adds its tile's qubits.  A write the engine
  // cannot follow makes it all ones; once the device pointer has been handed
  // out (`exposed`), writes through it cannot be followed at all.
  uint64_t support = 0;
  bool exposed = false;
  // plan cache for repeated circuit shapes (tiled mode; 0 entries = off)
  struct PlanEntry {
    std::vector<uint64_t> shape;              // the fused ops' shape words
    std::vector<DevOp> dops;                  // op program; matrices patched per use
    std::vector<int> src;                     // fused-op index of every dop
    std::vector<DevSegment> segs;
    std::vector<mlb::plan::PlannedPass> passes;
    cudaGraphExec_t exec = nullptr;           // the passes' launches, captured once
    void* graph_dplan = nullptr;              // d_plan the graph was captured with
    uint64_t last_use = 0;
  };
  std::vector<PlanEntry> plan_cache;
  size_t plan_cache_cap = 0;
  uint64_t plan_clock = 0;
  uint64_t plan_hits = 0, plan_misses = 0;
};

namespace {

// ---------------------------------------------------------------------------
// op validation and canonicalisation
// ---------------------------------------------------------------------------
bool is_zero(const double* m, int k) { return m[2 * k] == 0.0 && m[2 * k + 1] == 0.0; }
bool is_one(const double* m, int k) { return m[2 * k] == 1.0 && m[2 * k + 1] == 0.0; }

int validate(const mlb_state* s, const mlb_op_t& o) {
  const uint32_t n = s->n;
  const uint64_t all = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
  auto bad_q = [&](int q) { return q < 0 || (uint32_t)q >= n; };
  if (o.cmask & ~all) return fail(MLB_ERR_INVALID_QUBIT, "control mask outside the register");
  switch (o.kind) {
    case MLB_OP_1Q:
    case MLB_OP_X:
    case MLB_OP_DIAG1:
      if (bad_q(o.target)) return fail(MLB_ERR_INVALID_QUBIT, "target %d out of range", o.target);
      if (o.cmask >> o.target & 1ull) return fail(MLB_ERR_INVALID_QUBIT, "target in control mask");
      return MLB_OK;
    case MLB_OP_2Q:
    case MLB_OP_SWAP:
    case MLB_OP_ZZ:
      if (bad_q(o.target) || bad_q(o.target2))
        return fail(MLB_ERR_INVALID_QUBIT, "qubits (%d,%d) out of range", o.target, o.target2);
      if (o.target == o.target2) return fail(MLB_ERR_INVALID_QUBIT, "repeated qubit %d", o.target);
      if ((o.cmask >> o.target & 1ull) || (o.cmask >> o.target2 & 1ull))
        return fail(MLB_ERR_INVALID_QUBIT, "target in control mask");
      return MLB_OK;
    case MLB_OP_PHASE:
      if (o.cmask == 0) return fail(MLB_ERR_INVALID_ARG, "phase op with empty mask");
      return MLB_OK;
    default:
      return fail(MLB_ERR_INVALID_ARG, "unknown op kind %d", o.kind);
  }
}

// Rewrite an op into the cheapest equivalent kind.  Matrices are only
// re-labelled, never re-computed, so values stay bit-identical.
mlb_op_t canonical(const mlb_op_t& in) {
  mlb_op_t o = in;
  if (o.kind == MLB_OP_1Q) {
    const double* m = o.m;
    if (is_zero(m, 1) && is_zero(m, 2)) {  // diagonal
      mlb_op_t d{};
      d.kind = MLB_OP_DIAG1;
      d.target = o.target;
      d.target2 = -1;
      d.cmask = o.cmask;
      d.m[0] = m[0]; d.m[1] = m[1]; d.m[2] = m[6]; d.m[3] = m[7];
      if (is_one(d.m, 0)) {  // phase on the |1> half only
        mlb_op_t p{};
        p.kind = MLB_OP_PHASE;
        p.target = o.target;
        p.target2 = -1;
        p.cmask = o.cmask | (1ull << o.target);
        p.m[0] = m[6]; p.m[1] = m[7];
        return p;
      }
      return d;
    }
    if (is_zero(m, 0) && is_zero(m, 3) && is_one(m, 1) && is_one(m, 2)) {
      mlb_op_t x{};
      x.kind = MLB_OP_X;
      x.target = o.target;
      x.target2 = -1;
      x.cmask = o.cmask;
      return x;
    }
    return o;
  }
  if (o.kind == MLB_OP_2Q) {
    const double* m = o.m;  // m[(r*4+c)*2]
    auto E = [&](int r, int c) { return r * 4 + c; };
    bool diag = true;
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++)
        if (r != c && !is_zero(m, E(r, c))) diag = false;
    const int q0 = o.target, q1 = o.target2;
    if (diag) {
      if (is_one(m, E(0, 0)) && is_one(m, E(1, 1)) && is_one(m, E(2, 2))) {
        mlb_op_t p{};
        p.kind = MLB_OP_PHASE;
        p.target = q0;
        p.target2 = q1;
        p.cmask = o.cmask | (1ull << q0) | (1ull << q1);
        p.m[0] = m[2 * E(3, 3)]; p.m[1] = m[2 * E(3, 3) + 1];
        return p;
      }
      const double* a = &m[2 * E(0, 0)];
      const double* b = &m[2 * E(1, 1)];
      const double* c = &m[2 * E(2, 2)];
      const double* d = &m[2 * E(3, 3)];
      if (a[0] == d[0] && a[1] == d[1] && b[0] == c[0] && b[1] == c[1] && o.cmask == 0) {
        mlb_op_t z{};
        z.kind = MLB_OP_ZZ;
        z.target = q0;
        z.target2 = q1;
        z.m[0] = a[0]; z.m[1] = a[1]; z.m[2] = b[0]; z.m[3] = b[1];
        return z;
      }
    }
    // SWAP permutation
    bool swp = true;
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) {
        const int want = (r == 0 && c == 0) || (r == 3 && c == 3) || (r == 1 && c == 2) || (r == 2 && c == 1);
        if (want ? !is_one(m, E(r, c)) : !is_zero(m, E(r, c))) swp = false;
      }
    if (swp) {
      mlb_op_t w{};
      w.kind = MLB_OP_SWAP;
      w.target = q0;
      w.target2 = q1;
      w.cmask = o.cmask;
      return w;
    }
    // controlled-1q with control q0 (identity on the q0 = 0 sector, rows/cols 0 and 2)
    auto ctrl_form = [&](int i0, int i1, int j0, int j1) {
      // identity on indices i0,i1; zero couplings between {i0,i1} and {j0,j1}
      if (!is_one(m, E(i0, i0)) || !is_one(m, E(i1, i1))) return false;
      if (!is_zero(m, E(i0, i1)) || !is_zero(m, E(i1, i0))) return false;
      const int I[2] = {i0, i1}, J[2] = {j0, j1};
      for (int a2 = 0; a2 < 2; a2++)
        for (int b2 = 0; b2 < 2; b2++)
          if (!is_zero(m, E(I[a2], J[b2])) || !is_zero(m, E(J[b2], I[a2]))) return false;
      return true;
    };
    if (ctrl_form(0, 2, 1, 3)) {  // control q0, target q1, U from rows/cols {1,3}
      mlb_op_t u{};
      u.kind = MLB_OP_1Q;
      u.target = q1;
      u.target2 = -1;
      u.cmask = o.cmask | (1ull << q0);
      const int idx[4] = {E(1, 1), E(1, 3), E(3, 1), E(3, 3)};
      for (int k = 0; k < 4; k++) { u.m[2 * k] = m[2 * idx[k]]; u.m[2 * k + 1] = m[2 * idx[k] + 1]; }
      return canonical(u);
    }
    if (ctrl_form(0, 1, 2, 3)) {  // control q1, target q0, U from rows/cols {2,3}
      mlb_op_t u{};
      u.kind = MLB_OP_1Q;
      u.target = q0;
      u.target2 = -1;
      u.cmask = o.cmask | (1ull << q1);
      const int idx[4] = {E(2, 2), E(2, 3), E(3, 2), E(3, 3)};
      for (int k = 0; k < 4; k++) { u.m[2 * k] = m[2 * idx[k]]; u.m[2 * k + 1] = m[2 * idx[k] + 1]; }
      return canonical(u);
    }
    return o;
  }
  if (o.kind == MLB_OP_DIAG1 && is_one(o.m, 0)) {
    mlb_op_t p{};
    p.kind = MLB_OP_PHASE;
    p.target = o.target;
    p.target2 = -1;
    p.cmask = o.cmask | (1ull << o.target);
    p.m[0] = o.m[2]; p.m[1] = o.m[3];
    return p;
  }
  return o;
}

// Single-qubit op as a 2x2 matrix (for run fusion); false if not 1q-uncontrolled.
bool as_2x2(const mlb_op_t& o, double m[8]) {
  if (o.cmask != 0) {
    if (!(o.kind == MLB_OP_PHASE && popc(o.cmask) == 1)) return false;
  }
  switch (o.kind) {
    case MLB_OP_1Q: std::memcpy(m, o.m, 8 * sizeof(double)); return true;
    case MLB_OP_X: { const double x[8] = {0, 0, 1, 0, 1, 0, 0, 0}; std::memcpy(m, x, sizeof x); return true; }
    case MLB_OP_DIAG1: { const double d[8] = {o.m[0], o.m[1], 0, 0, 0, 0, o.m[2], o.m[3]}; std::memcpy(m, d, sizeof d); return true; }
    case MLB_OP_PHASE: { const double d[8] = {1, 0, 0, 0, 0, 0, o.m[0], o.m[1]}; std::memcpy(m, d, sizeof d); return true; }
    default: return false;
  }
}
int single_qubit_of(const mlb_op_t& o) {
  if (o.kind == MLB_OP_PHASE) return popc(o.cmask) == 1 ? __builtin_ctzll(o.cmask) : -1;
  if (o.cmask) return -1;
  if (o.kind == MLB_OP_1Q || o.kind == MLB_OP_X || o.kind == MLB_OP_DIAG1) return o.target;
  return -1;
}

// m = b * a (apply a first, then b)
void mul2(const double b[8], const double a[8], double out[8]) {
  for (int r = 0; r < 2; r++)
    for (int c = 0; c < 2; c++) {
      double re = 0, im = 0;
      for (int k = 0; k < 2; k++) {
        const double br = b[(r * 2 + k) * 2], bi = b[(r * 2 + k) * 2 + 1];
        const double ar = a[(k * 2 + c) * 2], ai = a[(k * 2 + c) * 2 + 1];
        re += br * ar - bi * ai;
        im += br * ai + bi * ar;
      }
      out[(r * 2 + c) * 2] = re;
      out[(r * 2 + c) * 2 + 1] = im;
    }
}

// Merge runs of uncontrolled single-qubit ops on the same qubit into one
// 2x2 (the FUSED_1Q rule of fuse_compile, fusion.c:247-292).
std::vector<mlb_op_t> fuse_1q_runs(const std::vector<mlb_op_t>& in, uint32_t n) {
  std::vector<mlb_op_t> out;
  out.reserve(in.size());
  std::vector<long> open(n, -1);  // index in out of the open 1q op per qubit
  for (const auto& o : in) {
    const int q = single_qubit_of(o);
    if (q >= 0 && open[q] >= 0) {
      double a[8], b[8], r[8];
      as_2x2(out[open[q]], a);
      as_2x2(o, b);
      mul2(b, a, r);
      mlb_op_t f{};
      f.kind = MLB_OP_1Q;
      f.target = q;
      f.target2 = -1;
      std::memcpy(f.m, r, sizeof r);
      out[open[q]] = f;
      continue;
    }
    const uint64_t qs = op_qubits(o);
    for (uint32_t b = 0; b < n; b++)
      if (qs >> b & 1ull) open[b] = -1;
    out.push_back(o);
    if (q >= 0) open[q] = (long)out.size() - 1;
  }
  for (auto& o : out)
    if (o.kind == MLB_OP_1Q) o = canonical(o);
  return out;
}

// X(t | c) . D . X(t | c), with D diagonal on t alone (a DIAG1 on t, or a
// phase on the |1> half of t) and the same single control c on both X's, is
// the parity phase d[bit t ^ bit c]: one ZZ op.  Each amplitude is
// multiplied by the same single diagonal entry as under the three ops (the
// X's only move amplitudes).  CNOT . RZ . CNOT is how the reference writes
// exp(-i g J Z Z) in QAOA's cost layer (qaoa.c:598-602, :750-753); as one
// diagonal op it needs no tile slot for its target.
std::vector<mlb_op_t> lift_parity_phases(const std::vector<mlb_op_t>& in) {
  std::vector<mlb_op_t> out;
  out.reserve(in.size());
  for (size_t i = 0; i < in.size(); i++) {
    if (i + 2 < in.size()) {
      const mlb_op_t &a = in[i], &d = in[i + 1], &b = in[i + 2];
      const int t = a.target;
      const bool cx = a.kind == MLB_OP_X && popc(a.cmask) == 1 && b.kind == MLB_OP_X && b.target == t &&
                      b.cmask == a.cmask;
      double dm[4];
      bool diag = false;
      if (cx && d.kind == MLB_OP_DIAG1 && d.target == t && d.cmask == 0) {
        std::memcpy(dm, d.m, sizeof dm);
        diag = true;
      } else if (cx && d.kind == MLB_OP_PHASE && d.cmask == (1ull << t)) {
        dm[0] = 1.0; dm[1] = 0.0; dm[2] = d.m[0]; dm[3] = d.m[1];
        diag = true;
      }
      if (diag) {
        mlb_op_t z{};
        z.kind = MLB_OP_ZZ;  // amp *= m[0..1] where bit target == bit target2, else m[2..3]
        z.target = __builtin_ctzll(a.cmask);
        z.target2 = t;
        std::memcpy(z.m, dm, sizeof dm);
        out.push_back(z);
        i += 2;
        continue;
      }
    }
    out.push_back(in[i]);
  }
  return out;
}

// The op-level fusion of a flush: 1-qubit runs, then CNOT . diagonal . CNOT
// sandwiches as parity phases.
std::vector<mlb_op_t> fuse_ops(const std::vector<mlb_op_t>& in, uint32_t n) {
  return lift_parity_phases(fuse_1q_runs(in, n));
}

int ensure_scratch(mlb_state* s, size_t bytes) {
  if (s->scratch_bytes >= bytes) return MLB_OK;
  if (s->d_scratch) {
    cudaStreamSynchronize(s->stream);
    cudaFree(s->d_scratch);
    s->d_scratch = nullptr;
    s->scratch_bytes = 0;
  }
  cudaError_t e = cudaMalloc((void**)&s->d_scratch, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "scratch allocation");
  s->scratch_bytes = bytes;
  return MLB_OK;
}

int upload_plan(mlb_state* s, const void* host, size_t bytes) {
  if (s->plan_ev_pending) {
    cudaEventSynchronize(s->plan_ev);
    s->plan_ev_pending = false;
  }
  if (s->h_plan_bytes < bytes) {
    if (s->h_plan) cudaFreeHost(s->h_plan);
    s->h_plan = nullptr;
    size_t nb = std::max(bytes, (size_t)1 << 20);
    cudaError_t e = cudaMallocHost(&s->h_plan, nb);
    if (e != cudaSuccess) { s->h_plan_bytes = 0; return cuda_fail(e, "pinned plan buffer"); }
    s->h_plan_bytes = nb;
  }
  if (s->d_plan_bytes < bytes) {
    if (s->d_plan) { cudaStreamSynchronize(s->stream); cudaFree(s->d_plan); }
    s->d_plan = nullptr;
    size_t nb = std::max(bytes, (size_t)1 << 20);
    cudaError_t e = cudaMalloc(&s->d_plan, nb);
    if (e != cudaSuccess) { s->d_plan_bytes = 0; return cuda_fail(e, "device plan buffer"); }
    s->d_plan_bytes = nb;
  }
  std::memcpy(s->h_plan, host, bytes);
  cudaError_t e = cudaMemcpyAsync(s->d_plan, s->h_plan, bytes, cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "plan upload");
  cudaEventRecord(s->plan_ev, s->stream);
  s->plan_ev_pending = true;
  return MLB_OK;
}

// Shape of a planned op list: everything the planner's decisions depend on
// (kind, qubits, controls, whether a 1-qubit matrix is real, and the dense
// setting), but not the matrix values.  Equal shapes plan identically.
std::vector<uint64_t> plan_shape(const mlb_state* s, const std::vector<mlb_op_t>& ops) {
  std::vector<uint64_t> w;
  w.reserve(2 * ops.size() + 1);
  w.push_back((uint64_t)s->n | (uint64_t)s->dtype << 8 | (uint64_t)s->dense_c128 << 16);
  for (const auto& o : ops) {
    uint64_t real = 0;
    if (o.kind == MLB_OP_1Q) {
      real = 1;
      for (int t = 1; t < 8; t += 2)
        if (o.m[t] != 0.0) real = 0;
    }
    w.push_back((uint64_t)(uint32_t)o.kind | (uint64_t)(uint8_t)o.target << 8 |
                (uint64_t)(uint8_t)o.target2 << 16 | real << 24);
    w.push_back(o.cmask);
  }
  return w;
}

// Fused complex64 path: dense <= 5-qubit blocks on the tensor cores.
int flush_fused(mlb_state* s, const std::vector<mlb_op_t>& ops, mlb_flush_stats_t& st) {
  fused::Plan P;
  int rc = fused::plan(ops, s->n, P);
  if (rc) return fail(rc, "fused path: an op spans more than 5 qubits or the state has < 13 qubits");
  if (!s->d_ferr) {
    cudaError_t e = cudaMalloc((void**)&s->d_ferr, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_ferr, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "fused error word");
  }
  // one upload: blocks, then operand images (16 KiB each, 16-byte aligned)
  const size_t bb = P.dev_blocks.size() * sizeof(FusedBlockDev);
  const size_t ioff = (bb + 255) & ~(size_t)255;
  std::vector<unsigned char> blob(ioff + P.images.size());
  std::memcpy(blob.data(), P.dev_blocks.data(), bb);
  std::memcpy(blob.data() + ioff, P.images.data(), P.images.size());
  rc = upload_plan(s, blob.data(), blob.size());
  if (rc) return rc;
  const FusedBlockDev* d_blocks = reinterpret_cast<const FusedBlockDev*>(s->d_plan);
  const uint8_t* d_images = reinterpret_cast<const uint8_t*>(s->d_plan) + ioff;
  cudaMemsetAsync(s->d_ferr, 0, sizeof(int), s->stream);
  const int skip = s->test_skip_copy ? 1 : 0;
  s->test_skip_copy = false;
  // all-zero tiles (see mlb_state::support): a pass runs over the tiles whose
  // outside bits may be nonzero, then adds its tile's qubits
  const uint64_t allq = s->n >= 64 ? ~0ull : ((1ull << s->n) - 1ull);
  const bool sparse = !s->exposed && (s->support & allq) != allq;
  uint64_t sup = s->support;
  for (size_t pi = 0; pi < P.dev_passes.size(); pi++) {
    FusedPassDev dp = P.dev_passes[pi];
    uint64_t tile = (1ull << dp.num_low) - 1ull;
    for (int h = 0; h < dp.num_high; h++) tile |= 1ull << dp.hbits[h];
    if (sparse) {
      const uint64_t fm = allq & ~tile & sup;
      dp.free_mask = (1ull << 63) | fm;
      dp.num_tiles = 1ull << popc(fm);
    }
    sup |= tile & allq;
    rc = launch_fused_pass(s->amp, (int)s->n, dp, d_blocks, d_images, s->d_ferr, s->num_sms, s->stream,
                           pi == 0 ? skip : 0);
    if (rc) { s->support = ~0ull; return fail(rc, "fused pass launch failed: %s", cudaGetErrorString(cudaGetLastError())); }
    st.passes++;
    st.kernel_launches++;
    st.bytes_moved += 2 * 8 * (dp.num_tiles << (dp.num_low + dp.num_high));
  }
  s->support = sup;
  cudaMemcpyAsync(s->h_ferr, s->d_ferr, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
  s->ferr_pending = true;
  st.ops += ops.size();
  st.dense_blocks += P.dev_blocks.size();
  st.segments += P.dev_blocks.size();
  return MLB_OK;
}

// Tile passes for ops (tiled mode, and the parts of a fused flush that need
// them), the plan taken from the state's plan cache when the shape repeats.
int flush_tiled(mlb_state* s, const std::vector<mlb_op_t>& ops, mlb_flush_stats_t& st) {
  const uint64_t dim = 1ull << s->n;
  const uint64_t ab = s->dtype == MLB_C128 ? 16 : 8;
  // the plan: from the cache when this shape ran before, else planned now
  mlb_state::PlanEntry local;
  mlb_state::PlanEntry* E = &local;
  bool hit = false;
  std::vector<uint64_t> shape;
  if (s->plan_cache_cap) {
    shape = plan_shape(s, ops);
    for (auto& e : s->plan_cache)
      if (e.shape == shape) {
        E = &e;
        hit = true;
        break;
      }
  }
  if (!hit) {
    Planner pl{s->n, s->dtype, geo(s->dtype)};
    pl.dense_limits = s->dtype == MLB_C128 && s->dense_c128;
    pl.plan(ops);
    local.dops = std::move(pl.dops);
    local.src = std::move(pl.dop_src);
    local.segs = std::move(pl.segs);
    local.passes = std::move(pl.passes);
    if (s->plan_cache_cap) {
      local.shape = std::move(shape);
      if (s->plan_cache.size() >= s->plan_cache_cap) {  // evict the least recently used
        auto lru = std::min_element(s->plan_cache.begin(), s->plan_cache.end(),
                                    [](const auto& a, const auto& b) { return a.last_use < b.last_use; });
        if (lru->exec) cudaGraphExecDestroy(lru->exec);
        s->plan_cache.erase(lru);
      }
      s->plan_cache.push_back(std::move(local));
      E = &s->plan_cache.back();
    }
    s->plan_misses++;
  } else {
    for (size_t i = 0; i < E->dops.size(); i++)  // this circuit's matrices into the cached program
      std::memcpy(E->dops[i].m, ops[E->src[i]].m, sizeof(E->dops[i].m));
    s->plan_hits++;
  }
  E->last_use = ++s->plan_clock;
  // complex128: register segments that fit run as dense 16x16 matrices on
  // the FP64 tensor cores (mode 2), built from this circuit's matrices every
  // flush; which segments fit depends only on the plan's shape, so the upload
  // layout (and a captured graph's pointers) repeat with the shape
  std::vector<DevSegment> dev_segs(E->segs);
  std::vector<DenseSegDev> dsegs;
  std::vector<dense::SegPlan> dplans;
  std::vector<int> dsrc;  // segment of each dense segment
  size_t nfrag = 0;
  if (s->dtype == MLB_C128 && s->dense_c128) {
    for (const auto& pp : E->passes)
      for (int k = 0; k < pp.pass.num_segments; k++) {
        const int si = pp.seg_begin + k;
        DenseSegDev D;
        dense::SegPlan S;
        if (dense::plan_segment(pp.pass, E->segs[si], E->dops.data(), D, S)) {
          D.frag_off = (uint32_t)nfrag;
          nfrag += (size_t)S.nvar * kDenseVarDoubles;
          dev_segs[si].mode = 2;
          dev_segs[si].dense = (int)dsegs.size();
          dsegs.push_back(D);
          dplans.push_back(S);
          dsrc.push_back(si);
        }
      }
  }
  // one upload: ops, segments, dense segments, dense fragments
  const size_t ob = E->dops.size() * sizeof(DevOp);
  const size_t sb = dev_segs.size() * sizeof(DevSegment);
  const size_t soff = (ob + 15) & ~(size_t)15;
  const size_t doff = (soff + sb + 15) & ~(size_t)15;
  const size_t foff = (doff + dsegs.size() * sizeof(DenseSegDev) + 15) & ~(size_t)15;
  const size_t total = foff + nfrag * sizeof(double);
  std::unique_ptr<unsigned char[]> blob(new unsigned char[total]);
  std::memset(blob.get(), 0, foff);
  std::memcpy(blob.get(), E->dops.data(), ob);
  std::memcpy(blob.get() + soff, dev_segs.data(), sb);
  if (!dsegs.empty()) {
    std::memcpy(blob.get() + doff, dsegs.data(), dsegs.size() * sizeof(DenseSegDev));
    // the segment matrices, in parallel over segments (~1 ms of host time each
    // for 64 variants)
    double* fr = reinterpret_cast<double*>(blob.get() + foff);
    std::atomic<size_t> next{0};
    auto work = [&]() {
      for (size_t k; (k = next.fetch_add(1)) < dsegs.size();)
        dense::fill_fragments(E->segs[dsrc[k]], E->dops.data(), dsegs[k], dplans[k], fr + dsegs[k].frag_off);
    };
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nth = std::min<size_t>({hw, (size_t)16, 1 + nfrag / (256 * 1024)});
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nth; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
  }
  int rc = upload_plan(s, blob.get(), total);
  if (rc) return rc;
  const DevOp* d_ops = reinterpret_cast<const DevOp*>(s->d_plan);
  const DevSegment* d_segs = reinterpret_cast<const DevSegment*>((unsigned char*)s->d_plan + soff);
  const DenseSegDev* d_dsegs = reinterpret_cast<const DenseSegDev*>((unsigned char*)s->d_plan + doff);
  const double* d_frags = reinterpret_cast<const double*>((unsigned char*)s->d_plan + foff);
  // Tiles that may hold nonzero amplitudes (see mlb_state::support): while
  // some qubit has not been touched since a reset, a pass runs only over the
  // tiles whose outside bits are touched ones.  Such launches depend on the
  // state's history, so they are never captured into a cached graph.
  const uint64_t allq = s->n >= 64 ? ~0ull : ((1ull << s->n) - 1ull);
  const bool sparse = !s->exposed && (s->support & allq) != allq;
  // until every launch went out, nothing is assumed about the state's zeros
  const uint64_t sup0 = s->support;
  s->support = ~0ull;
  // HBM bytes and dense-segment amplitude applications of the launches
  uint64_t moved = 0, dense_amps = 0;
  auto launch_passes = [&](bool restrict) -> int {
    uint64_t sup = sup0;
    moved = dense_amps = 0;
    for (const auto& pp : E->passes) {
      bool all_dense = pp.pass.num_segments > 0;
      int ndense = 0;
      for (int k = 0; k < pp.pass.num_segments; k++) {
        all_dense = all_dense && dev_segs[pp.seg_begin + k].mode == 2;
        ndense += dev_segs[pp.seg_begin + k].mode == 2;
      }
      DevPass pass = pp.pass;
      if (restrict) {
        pass.tile_free_mask &= sup;
        pass.num_tiles = 1ull << popc(pass.tile_free_mask);
        sup |= allq & ~pp.pass.tile_free_mask;  // this pass's tile qubits
      }
      const uint64_t amps = pass.num_tiles << (pass.L + pass.H);
      moved += 2 * ab * amps;
      dense_amps += (uint64_t)ndense * amps;
      const int r = launch_tile_pass(s->dtype, s->amp, pass, d_segs + pp.seg_begin, d_ops, d_dsegs, d_frags,
                                     s->num_sms, s->stream, all_dense);
      if (r) return r;
    }
    return MLB_OK;
  };
  if (sparse) {
    if ((rc = launch_passes(true))) return fail(rc, "tile pass launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  } else if (s->plan_cache_cap && E != &local) {
    // replay the captured launches (capture once per plan buffer)
    if (E->exec && E->graph_dplan != s->d_plan) {
      cudaGraphExecDestroy(E->exec);
      E->exec = nullptr;
    }
    if (!E->exec) {
      prepare_tile_launch(s->dtype);  // function attributes before capture
      cudaGraph_t g = nullptr;
      bool ok = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        const int lr = launch_passes(false);
        ok = cudaStreamEndCapture(s->stream, &g) == cudaSuccess && lr == MLB_OK && g;
        if (ok) ok = cudaGraphInstantiate(&E->exec, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
      }
      if (!ok) {
        cudaGetLastError();
        E->exec = nullptr;
      }
      E->graph_dplan = s->d_plan;
    }
    if (E->exec) {
      if (cudaGraphLaunch(E->exec, s->stream) != cudaSuccess)
        return fail(MLB_ERR_DRIVER, "graph launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    } else if ((rc = launch_passes(false))) {
      return fail(rc, "tile pass launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
  } else if ((rc = launch_passes(false))) {
    return fail(rc, "tile pass launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  s->support = sup0;
  for (const auto& pp : E->passes) s->support |= allq & ~pp.pass.tile_free_mask;
  if (!sparse) {  // every tile of every pass (a replayed graph runs no launch_passes)
    moved = E->passes.size() * 2 * ab * dim;
    dense_amps = dsegs.size() << s->n;
  }
  st.passes += E->passes.size();
  st.kernel_launches += E->passes.size();
  st.bytes_moved += moved;
  st.dense_amps += dense_amps;
  st.ops += ops.size();
  st.segments += E->segs.size();
  st.dense_blocks += dsegs.size();
  st.plan_cache_hit = hit ? 1 : 0;
  return MLB_OK;
}

int flush_impl(mlb_state* s) {
  if (s->queue.empty()) return MLB_OK;
  DeviceGuard dg(s->device);
  mlb_flush_stats_t st{};
  const uint64_t dim = 1ull << s->n;
  const uint64_t ab = s->dtype == MLB_C128 ? 16 : 8;
  if (s->mode == MLB_EXEC_EAGER) {
    if (s->timing) cudaEventRecord(s->t0, s->stream);
    for (const auto& o : s->queue) {
      int rc = launch_gate(s->dtype, s->amp, (int)s->n, o, s->stream);
      if (rc) { s->queue.clear(); s->support = ~0ull; return fail(rc, "gate launch failed: %s", cudaGetErrorString(cudaGetLastError())); }
      s->support |= op_targets(o);  // a gate mixes amplitudes that differ in its targets only
      st.ops++;
      st.passes++;
      st.kernel_launches++;
      const int c = popc(o.cmask);
      uint64_t touched = dim >> c;
      if (o.kind == MLB_OP_PHASE) touched = dim >> popc(o.cmask);
      st.bytes_moved += 2 * ab * touched;
    }
    s->queue.clear();
    if (s->timing) {
      cudaEventRecord(s->t1, s->stream);
      s->timed_pending = true;
    }
    s->stats = st;
    return MLB_OK;
  }
  std::vector<mlb_op_t> ops = s->fuse1q ? fuse_ops(s->queue, s->n) : s->queue;
  s->queue.clear();
  if (s->timing) cudaEventRecord(s->t0, s->stream);
  int rc = MLB_OK;
  if (s->mode != MLB_EXEC_FUSED || s->n < (uint32_t)fused::kTileBits) {
    rc = flush_tiled(s, ops, st);
  } else {
    // fused blocks for runs of ops on <= 5 qubits; a wider op (a many-
    // controlled gate) runs as a tile pass between them, in order
    size_t i = 0;
    while (!rc && i < ops.size()) {
      size_t j = i;
      const bool wide = popc(op_qubits(ops[i])) > fused::kBlockQubits;
      while (j < ops.size() && (popc(op_qubits(ops[j])) > fused::kBlockQubits) == wide) j++;
      const std::vector<mlb_op_t> run(ops.begin() + i, ops.begin() + j);
      rc = wide ? flush_tiled(s, run, st) : flush_fused(s, run, st);
      i = j;
    }
  }
  if (rc) return rc;
  if (s->timing) {
    cudaEventRecord(s->t1, s->stream);
    s->timed_pending = true;
  }
  s->stats = st;
  return MLB_OK;
}

int enqueue(mlb_state* s, const mlb_op_t& op) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  int rc = validate(s, op);
  if (rc) return rc;
  s->queue.push_back(canonical(op));
  if (s->queue.size() >= 65536) return flush_impl(s);
  return MLB_OK;
}

int sync_stream(mlb_state* s) {
  cudaError_t e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
  if (s->ferr_pending) {
    s->ferr_pending = false;
    if (*s->h_ferr) return fail(MLB_ERR_TIMEOUT, "fused pass: tensor-core completion wait ran out");
  }
  return MLB_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* mlb_status_string(int st) {
  switch (st) {
    case MLB_OK: return "ok";
    case MLB_ERR_OUT_OF_MEMORY: return "out of device memory";
    case MLB_ERR_NO_DEVICE: return "no CUDA device";
    case MLB_ERR_DRIVER: return "CUDA driver/runtime error";
    case MLB_ERR_INVALID_QUBIT: return "invalid qubit";
    case MLB_ERR_NUM_QUBITS: return "unsupported number of qubits";
    case MLB_ERR_INVALID_ARG: return "invalid argument";
    case MLB_ERR_TIMEOUT: return "device wait timed out";
    case MLB_ERR_BUSY: return "admission refused";
    case MLB_ERR_NOT_SUPPORTED: return "not supported";
    default: return "unknown status";
  }
}

const char* mlb_last_error(void) { return g_err.c_str(); }

int mlb_device_count(int* count) {
  if (!count) return fail(MLB_ERR_INVALID_ARG, "null count");
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    *count = 0;
    cudaGetLastError();
    return fail(MLB_ERR_NO_DEVICE, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
  }
  *count = c;
  return MLB_OK;
}

int mlb_fp64_tensor_peak(int device, double* tflops) {
  if (!tflops) return fail(MLB_ERR_INVALID_ARG, "null out");
  int cnt = 0;
  if (mlb_device_count(&cnt) != MLB_OK || device < 0 || device >= cnt) return fail(MLB_ERR_NO_DEVICE, "no such device");
  DeviceGuard dg(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (sms < 1) return fail(MLB_ERR_DRIVER, "multiprocessor count");
  const int rc = measure_fp64_tensor_peak(sms, tflops);
  return rc ? fail(rc, "fp64 tensor probe") : MLB_OK;
}

int mlb_state_create(uint32_t n, int dtype, int device, mlb_state_t** out) {
  if (!out) return fail(MLB_ERR_INVALID_ARG, "null out");
  *out = nullptr;
  if (dtype != MLB_C128 && dtype != MLB_C64) return fail(MLB_ERR_INVALID_ARG, "bad dtype %d", dtype);
  const uint32_t maxq = dtype == MLB_C128 ? 33 : 34;
  if (n < 1 || n > maxq) return fail(MLB_ERR_NUM_QUBITS, "num_qubits %u outside [1, %u]", n, maxq);
  int cnt = 0;
  if (mlb_device_count(&cnt) != MLB_OK || cnt == 0) return fail(MLB_ERR_NO_DEVICE, "no CUDA device visible");
  if (device < 0 || device >= cnt) return fail(MLB_ERR_NO_DEVICE, "device %d of %d", device, cnt);
  DeviceGuard dg(device);
  auto* s = new (std::nothrow) mlb_state();
  if (!s) return fail(MLB_ERR_OUT_OF_MEMORY, "host allocation");
  s->n = n;
  s->dtype = dtype;
  s->device = device;
  // complex64 states run the fused tensor-core path by default (states under
  // 13 qubits fall back to tile passes inside the flush)
  s->mode = dtype == MLB_C64 ? MLB_EXEC_FUSED : MLB_EXEC_TILED;
  s->bytes = (size_t)(dtype == MLB_C128 ? 16 : 8) << n;
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaError_t e = cudaMalloc(&s->amp, s->bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return cuda_fail(e, "state allocation");
  }
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->plan_ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cudaFree(s->amp);
    delete s;
    return cuda_fail(e, "stream creation");
  }
  int rc = launch_init_zero(dtype, s->amp, (int)n, s->stream);
  if (rc) {
    mlb_state_free(s);
    return fail(rc, "init kernel");
  }
  s->support = 0;  // |0...0>
  *out = s;
  return MLB_OK;
}

void mlb_state_free(mlb_state_t* s) {
  if (!s) return;
  DeviceGuard dg(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->amp) cudaFree(s->amp);
  if (s->d_scratch) cudaFree(s->d_scratch);
  if (s->d_plan) cudaFree(s->d_plan);
  for (auto& e : s->plan_cache)
    if (e.exec) cudaGraphExecDestroy(e.exec);
  if (s->d_ferr) cudaFree(s->d_ferr);
  if (s->h_ferr) cudaFreeHost(s->h_ferr);
  if (s->h_plan) cudaFreeHost(s->h_plan);
  if (s->plan_ev) cudaEventDestroy(s->plan_ev);
  if (s->t0) cudaEventDestroy(s->t0);
  if (s->t1) cudaEventDestroy(s->t1);
  if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
  delete s;
}

int mlb_state_num_qubits(const mlb_state_t* s, uint32_t* out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  *out = s->n;
  return MLB_OK;
}
int mlb_state_dim(const mlb_state_t* s, uint64_t* out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  *out = 1ull << s->n;
  return MLB_OK;
}
int mlb_state_dtype(const mlb_state_t* s, int* out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  *out = s->dtype;
  return MLB_OK;
}
int mlb_state_device_ptr(mlb_state_t* s, void** out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  int rc = flush_impl(s);
  if (rc) return rc;
  s->exposed = true;  // writes through the pointer cannot be followed
  s->support = ~0ull;
  *out = s->amp;
  return MLB_OK;
}
int mlb_state_set_stream(mlb_state_t* s, void* stream) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  rc = sync_stream(s);
  if (rc) return rc;
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  if (stream) {
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
  } else {
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "stream creation");
    s->own_stream = true;
  }
  return MLB_OK;
}
int mlb_state_stream(const mlb_state_t* s, void** out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  *out = (void*)s->stream;
  return MLB_OK;
}
int mlb_test_fused_skip_copy(mlb_state_t* s) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  if (s->dtype != MLB_C64) return fail(MLB_ERR_NOT_SUPPORTED, "the fused path runs complex64 states");
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);  // queued ops run as they were queued
  if (rc) return rc;
  s->test_skip_copy = true;
  return MLB_OK;
}

int mlb_state_set_dense(mlb_state_t* s, int on) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);  // queued ops keep the setting they were queued under
  if (rc) return rc;
  if (s->dense_c128 != (on != 0)) {
    rc = sync_stream(s);  // cached graphs read the old segment modes; they may still be running
    if (rc) return rc;
    for (auto& e : s->plan_cache)
      if (e.exec) {
        cudaGraphExecDestroy(e.exec);
        e.exec = nullptr;
      }
  }
  s->dense_c128 = on != 0;
  return MLB_OK;
}

int mlb_state_set_plan_cache(mlb_state_t* s, size_t entries) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  if (entries < s->plan_cache.size()) {
    rc = sync_stream(s);  // graphs may still be running
    if (rc) return rc;
    for (auto& e : s->plan_cache)
      if (e.exec) cudaGraphExecDestroy(e.exec);
    s->plan_cache.clear();
  }
  s->plan_cache_cap = entries;
  return MLB_OK;
}

int mlb_state_set_exec_mode(mlb_state_t* s, int mode) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  if (mode != MLB_EXEC_TILED && mode != MLB_EXEC_EAGER && mode != MLB_EXEC_FUSED)
    return fail(MLB_ERR_NOT_SUPPORTED, "exec mode %d not available", mode);
  if (mode == MLB_EXEC_FUSED && s->dtype != MLB_C64)
    return fail(MLB_ERR_NOT_SUPPORTED, "the fused path runs on complex64 states");
  int rc = flush_impl(s);
  if (rc) return rc;
  s->mode = mode;
  return MLB_OK;
}
int mlb_state_reset(mlb_state_t* s) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  DeviceGuard dg(s->device);
  s->queue.clear();
  const int rc = launch_init_zero(s->dtype, s->amp, (int)s->n, s->stream);
  s->support = rc ? ~0ull : 0;  // |0...0>
  return rc;
}
int mlb_state_copy_to_host(mlb_state_t* s, void* host) {
  if (!s || !host) return fail(MLB_ERR_INVALID_ARG, "null argument");
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(host, s->amp, s->bytes, cudaMemcpyDeviceToHost, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "copy to host");
  return sync_stream(s);
}
int mlb_state_copy_from_host(mlb_state_t* s, const void* host) {
  if (!s || !host) return fail(MLB_ERR_INVALID_ARG, "null argument");
  DeviceGuard dg(s->device);
  s->queue.clear();  // the upload overwrites whatever was pending
  s->support = ~0ull;
  cudaError_t e = cudaMemcpyAsync(s->amp, host, s->bytes, cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "copy from host");
  return sync_stream(s);
}
int mlb_state_copy(mlb_state_t* dst, mlb_state_t* src) {
  if (!dst || !src) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (dst->n != src->n) return fail(MLB_ERR_INVALID_ARG, "qubit counts differ");
  int rc = flush_impl(src);
  if (rc) return rc;
  dst->queue.clear();
  dst->support = src->exposed ? ~0ull : src->support;
  DeviceGuard dg(dst->device);
  rc = sync_stream(src);
  if (rc) return rc;
  if (dst->dtype == src->dtype) {
    cudaError_t e = cudaMemcpyAsync(dst->amp, src->amp, src->bytes, cudaMemcpyDeviceToDevice, dst->stream);
    if (e != cudaSuccess) return cuda_fail(e, "state copy");
  } else {
    rc = launch_convert(dst->dtype, dst->amp, src->dtype, src->amp, 1ull << src->n, dst->stream);
    if (rc) return fail(rc, "convert kernel");
  }
  return sync_stream(dst);
}
int mlb_flush(mlb_state_t* s) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  return flush_impl(s);
}
int mlb_synchronize(mlb_state_t* s) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  int rc = flush_impl(s);
  if (rc) return rc;
  DeviceGuard dg(s->device);
  return sync_stream(s);
}

// ---- gates ----------------------------------------------------------------
int mlb_apply_op(mlb_state_t* s, const mlb_op_t* op) {
  if (!s || !op) return fail(MLB_ERR_INVALID_ARG, "null argument");
  return enqueue(s, *op);
}
int mlb_apply_ops(mlb_state_t* s, const mlb_op_t* ops, size_t num) {
  if (!s || (!ops && num)) return fail(MLB_ERR_INVALID_ARG, "null argument");
  for (size_t i = 0; i < num; i++) {
    int rc = enqueue(s, ops[i]);
    if (rc) return rc;
  }
  return MLB_OK;
}
int mlb_apply_1q(mlb_state_t* s, uint32_t t, const double m[8]) {
  if (!m) return fail(MLB_ERR_INVALID_ARG, "null matrix");
  mlb_op_t o{};
  o.kind = MLB_OP_1Q;
  o.target = (int)t;
  o.target2 = -1;
  std::memcpy(o.m, m, 8 * sizeof(double));
  return enqueue(s, o);
}
int mlb_apply_2q(mlb_state_t* s, uint32_t q0, uint32_t q1, const double m[32]) {
  if (!m) return fail(MLB_ERR_INVALID_ARG, "null matrix");
  mlb_op_t o{};
  o.kind = MLB_OP_2Q;
  o.target = (int)q0;
  o.target2 = (int)q1;
  std::memcpy(o.m, m, 32 * sizeof(double));
  return enqueue(s, o);
}
int mlb_apply_controlled_1q(mlb_state_t* s, uint64_t cmask, uint32_t t, const double m[8]) {
  if (!m) return fail(MLB_ERR_INVALID_ARG, "null matrix");
  mlb_op_t o{};
  o.kind = MLB_OP_1Q;
  o.target = (int)t;
  o.target2 = -1;
  o.cmask = cmask;
  std::memcpy(o.m, m, 8 * sizeof(double));
  return enqueue(s, o);
}
int mlb_apply_mcx(mlb_state_t* s, uint64_t cmask, uint32_t t) {
  mlb_op_t o{};
  o.kind = MLB_OP_X;
  o.target = (int)t;
  o.target2 = -1;
  o.cmask = cmask;
  return enqueue(s, o);
}
int mlb_apply_mcz(mlb_state_t* s, uint64_t all_mask) {
  mlb_op_t o{};
  o.kind = MLB_OP_PHASE;
  o.target = all_mask ? __builtin_ctzll(all_mask) : 0;
  o.target2 = -1;
  o.cmask = all_mask;
  o.m[0] = -1.0;
  o.m[1] = 0.0;
  return enqueue(s, o);
}
int mlb_apply_swap(mlb_state_t* s, uint64_t cmask, uint32_t q0, uint32_t q1) {
  mlb_op_t o{};
  o.kind = MLB_OP_SWAP;
  o.target = (int)q0;
  o.target2 = (int)q1;
  o.cmask = cmask;
  return enqueue(s, o);
}
int mlb_apply_zz(mlb_state_t* s, uint32_t q0, uint32_t q1, double theta) {
  mlb_op_t o{};
  o.kind = MLB_OP_ZZ;
  o.target = (int)q0;
  o.target2 = (int)q1;
  mlb_mat_zz(theta, o.m);
  return enqueue(s, o);
}

// ---- reductions -----------------------------------------------------------
static int probs_z(mlb_state_t* s, std::vector<double>& out) {
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  const uint64_t dim = 1ull << s->n;
  const uint64_t chunks = s->n >= 13 ? dim >> 13 : 1;
  const size_t need = sizeof(double) * ((size_t)s->num_sms * 4 * 14 + chunks + 64 + 64);
  rc = ensure_scratch(s, need);
  if (rc) return rc;
  double* d_out = s->d_scratch;
  rc = launch_reduce_probs_z(s->dtype, s->amp, (int)s->n, d_out, s->d_scratch + 64, s->num_sms, s->stream);
  if (rc) return fail(rc, "reduction launch");
  out.assign(s->n + 1, 0.0);
  cudaError_t e = cudaMemcpyAsync(out.data(), d_out, (s->n + 1) * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "reduction readback");
  return sync_stream(s);
}

int mlb_norm_sq(mlb_state_t* s, double* out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  std::vector<double> v;
  int rc = probs_z(s, v);
  if (rc) return rc;
  *out = v[s->n];
  return MLB_OK;
}
int mlb_prob_one_all(mlb_state_t* s, double* out_n) {
  if (!s || !out_n) return fail(MLB_ERR_INVALID_ARG, "null argument");
  std::vector<double> v;
  int rc = probs_z(s, v);
  if (rc) return rc;
  std::memcpy(out_n, v.data(), s->n * sizeof(double));
  return MLB_OK;
}
int mlb_prob_one(mlb_state_t* s, uint32_t q, double* out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (q >= s->n) return fail(MLB_ERR_INVALID_QUBIT, "qubit %u", q);
  std::vector<double> v;
  int rc = probs_z(s, v);
  if (rc) return rc;
  *out = v[q];
  return MLB_OK;
}
static int seq_sum(mlb_state_t* s, uint64_t fmask, uint64_t fval, bool fused, double* total);

int mlb_prob_one_exact(mlb_state_t* s, uint32_t q, double* out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (q >= s->n) return fail(MLB_ERR_INVALID_QUBIT, "qubit %u", q);
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  return seq_sum(s, 1ull << q, 1ull << q, true, out);
}
int mlb_expect_z_all(mlb_state_t* s, double* out_n) {
  int rc = mlb_prob_one_all(s, out_n);
  if (rc) return rc;
  for (uint32_t q = 0; q < s->n; q++) out_n[q] = 1.0 - 2.0 * out_n[q];
  return MLB_OK;
}

int mlb_expect_pauli_sum(mlb_state_t* s, size_t num_terms, const uint64_t* xm, const uint64_t* zm,
                         const double* coeffs, double* out) {
  if (!s || !out || (num_terms && (!xm || !zm))) return fail(MLB_ERR_INVALID_ARG, "null argument");
  const uint64_t allm = s->n >= 64 ? ~0ull : ((1ull << s->n) - 1ull);
  for (size_t t = 0; t < num_terms; t++)
    if ((xm[t] | zm[t]) & ~allm) return fail(MLB_ERR_INVALID_QUBIT, "Pauli term %zu outside the register", t);
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  // group terms by X mask (<= 16 per launch)
  std::vector<size_t> order(num_terms);
  for (size_t i = 0; i < num_terms; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return xm[a] < xm[b]; });
  const size_t need = sizeof(double) * ((size_t)s->num_sms * 8 * 16 + 64) + 64 * (sizeof(uint64_t) + sizeof(int)) + 256;
  rc = ensure_scratch(s, need);
  if (rc) return rc;
  std::vector<double> vals(num_terms, 0.0);
  double* d_terms = s->d_scratch;
  uint64_t* d_z = reinterpret_cast<uint64_t*>(s->d_scratch + 16);
  int* d_ny = reinterpret_cast<int*>(s->d_scratch + 32);
  double* d_parts = s->d_scratch + 64;
  size_t i = 0;
  while (i < num_terms) {
    const uint64_t x = xm[order[i]];
    size_t j = i;
    uint64_t hz[16];
    int hny[16];
    while (j < num_terms && xm[order[j]] == x && j - i < 16) {
      hz[j - i] = zm[order[j]];
      hny[j - i] = popc(xm[order[j]] & zm[order[j]]);
      j++;
    }
    const int cnt = (int)(j - i);
    cudaMemcpyAsync(d_z, hz, cnt * sizeof(uint64_t), cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(d_ny, hny, cnt * sizeof(int), cudaMemcpyHostToDevice, s->stream);
    rc = launch_pauli_group(s->dtype, s->amp, (int)s->n, x, cnt, d_z, d_ny, d_terms, d_parts, s->num_sms, s->stream);
    if (rc) return fail(rc, "pauli launch");
    double hv[16];
    cudaMemcpyAsync(hv, d_terms, cnt * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    rc = sync_stream(s);
    if (rc) return rc;
    for (int k = 0; k < cnt; k++) vals[order[i + k]] = hv[k];
    i = j;
  }
  double acc = 0.0;
  for (size_t t = 0; t < num_terms; t++) acc += (coeffs ? coeffs[t] : 1.0) * vals[t];
  *out = acc;
  return MLB_OK;
}
int mlb_expect_pauli(mlb_state_t* s, uint64_t xmask, uint64_t zmask, double* out) {
  const double one = 1.0;
  return mlb_expect_pauli_sum(s, 1, &xmask, &zmask, &one, out);
}
int mlb_correlation_zz(mlb_state_t* s, uint32_t q1, uint32_t q2, double* out) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  if (q1 >= s->n || q2 >= s->n) return fail(MLB_ERR_INVALID_QUBIT, "qubit out of range");
  const uint64_t z = (1ull << q1) ^ (1ull << q2);
  return mlb_expect_pauli(s, 0, z, out);
}

int mlb_probabilities(mlb_state_t* s, int rule, double* out_host, void* out_device) {
  if (!s || (!out_host && !out_device)) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (rule != 0 && rule != 1) return fail(MLB_ERR_INVALID_ARG, "rule %d", rule);
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  const uint64_t dim = 1ull << s->n;
  double* dst = (double*)out_device;
  bool temp = false;
  if (!dst) {
    cudaError_t e = cudaMallocAsync((void**)&dst, dim * sizeof(double), s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "probability buffer");
    temp = true;
  }
  rc = launch_probabilities(s->dtype, s->amp, (int)s->n, rule, dst, s->stream);
  if (rc) return fail(rc, "probability kernel");
  if (out_host) {
    cudaError_t e = cudaMemcpyAsync(out_host, dst, dim * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "probability readback");
  }
  if (temp) cudaFreeAsync(dst, s->stream);
  return sync_stream(s);
}

// ---- sampling / collapse ---------------------------------------------------
int mlb_sample(mlb_state_t* s, int rule, const double* u, size_t num, uint64_t* out) {
  if (!s || (num && (!u || !out))) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (rule != MLB_SAMPLE_CDF_GE && rule != MLB_SAMPLE_CUM_GT) return fail(MLB_ERR_INVALID_ARG, "rule %d", rule);
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  char eb[8];
  rc = sample_exact(s->dtype, s->amp, (int)s->n, rule, u, num, out, s->num_sms, s->stream, eb, sizeof eb);
  if (rc) return fail(rc, "sampling: %s", cudaGetErrorString(cudaGetLastError()));
  return MLB_OK;
}

static int seq_sum(mlb_state_t* s, uint64_t fmask, uint64_t fval, bool fused, double* total) {
  int rc = seq_sum_exact(s->dtype, s->amp, (int)s->n, fmask, fval, fused, s->num_sms, s->stream, total);
  if (rc) return fail(rc, "sequential sum: %s", cudaGetErrorString(cudaGetLastError()));
  return MLB_OK;
}

int mlb_measure_qubit(mlb_state_t* s, uint32_t q, double u, int* outcome) {
  if (!s || !outcome) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (q >= s->n) return fail(MLB_ERR_INVALID_QUBIT, "qubit %u", q);
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  const uint64_t b = 1ull << q;
  // measurement_probability_one and the kept-half norm both accumulate with
  // fused multiply-adds in the reference build (measurement.c:93, :214).
  double p1 = 0.0;
  rc = seq_sum(s, b, b, true, &p1);
  if (rc) return rc;
  const int r = (u < p1) ? 1 : 0;
  double nf = p1;
  if (r == 0) {
    rc = seq_sum(s, b, 0, true, &nf);
    if (rc) return rc;
  }
  if (nf <= 1e-15) {  // zero the other half, leave unnormalised (measurement.c:222-231)
    rc = launch_scale(s->dtype, s->amp, (int)s->n, 1.0, b, r ? b : 0, s->stream);
    if (rc) return fail(rc, "collapse kernel");
    *outcome = -1;
    return sync_stream(s);
  }
  const double inv = 1.0 / std::sqrt(nf);
  rc = launch_scale(s->dtype, s->amp, (int)s->n, inv, b, r ? b : 0, s->stream);
  if (rc) return fail(rc, "collapse kernel");
  *outcome = r;
  return sync_stream(s);
}

int mlb_quantum_measure(mlb_state_t* s, uint32_t q, double u, int* outcome, double* probability) {
  if (!s || !outcome) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (q >= s->n) return fail(MLB_ERR_INVALID_QUBIT, "qubit %u", q);
  DeviceGuard dg(s->device);
  int rc = flush_impl(s);
  if (rc) return rc;
  const uint64_t b = 1ull << q;
  double p0 = 0.0, p1 = 0.0;
  // quantum_measure rounds product and sum separately (gates.c:1150-1199).
  if ((rc = seq_sum(s, b, 0, false, &p0))) return rc;
  if ((rc = seq_sum(s, b, b, false, &p1))) return rc;
  const int r = (u < p0) ? 0 : 1;
  const double keep = r == 0 ? p0 : p1;
  if (probability) *probability = keep;
  if (keep <= 1e-15) {  // gates.c:1203-1205: dropped half zeroed, result {0, 0}
    rc = launch_scale(s->dtype, s->amp, (int)s->n, 1.0, b, r ? b : 0, s->stream);
    if (rc) return fail(rc, "collapse kernel");
    *outcome = 0;
    if (probability) *probability = 0.0;
    return sync_stream(s);
  }
  const double nrm = std::sqrt(keep);
  rc = launch_scale(s->dtype, s->amp, (int)s->n, -nrm, b, r ? b : 0, s->stream);  // divide
  if (rc) return fail(rc, "collapse kernel");
  *outcome = r;
  return sync_stream(s);
}

int mlb_measure_all(mlb_state_t* s, double u, uint64_t* outcome) {
  if (!s || !outcome) return fail(MLB_ERR_INVALID_ARG, "null argument");
  int rc = mlb_sample(s, MLB_SAMPLE_CUM_GT, &u, 1, outcome);
  if (rc) return rc;
  DeviceGuard dg(s->device);
  // collapse to |outcome>: zero everything, then write 1 at the index
  s->support = ~0ull;
  cudaError_t e = cudaMemsetAsync(s->amp, 0, s->bytes, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "collapse memset");
  if (s->dtype == MLB_C128) {
    const double one[2] = {1.0, 0.0};
    e = cudaMemcpyAsync((char*)s->amp + 16 * (*outcome), one, 16, cudaMemcpyHostToDevice, s->stream);
  } else {
    const float one[2] = {1.0f, 0.0f};
    e = cudaMemcpyAsync((char*)s->amp + 8 * (*outcome), one, 8, cudaMemcpyHostToDevice, s->stream);
  }
  if (e != cudaSuccess) return cuda_fail(e, "collapse write");
  rc = sync_stream(s);
  if (!rc) s->support = *outcome;  // only amplitude `outcome` is nonzero
  return rc;
}

int mlb_normalize(mlb_state_t* s, double* norm_out) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  double nsq = 0.0;
  int rc = mlb_norm_sq(s, &nsq);
  if (rc) return rc;
  const double nrm = std::sqrt(nsq);
  if (norm_out) *norm_out = nrm;
  if (nrm < 1e-15) return fail(MLB_ERR_INVALID_ARG, "state norm %g too small to normalise", nrm);
  DeviceGuard dg(s->device);
  rc = launch_scale(s->dtype, s->amp, (int)s->n, -nrm, 0, 0, s->stream);
  if (rc) return fail(rc, "normalise kernel");
  return sync_stream(s);
}

// ---- circuits -------------------------------------------------------------
int mlb_gates_to_ops(const mlb_gate_t* gates, size_t num, uint32_t n, mlb_op_t* ops, size_t* num_ops) {
  if ((!gates && num) || !num_ops) return fail(MLB_ERR_INVALID_ARG, "null argument");
  size_t k = 0;
  auto emit = [&](const mlb_op_t& o) {
    if (ops) ops[k] = o;
    k++;
  };
  auto one = [&](int t, const double m[8]) {
    mlb_op_t o{};
    o.kind = MLB_OP_1Q;
    o.target = t;
    o.target2 = -1;
    std::memcpy(o.m, m, 8 * sizeof(double));
    emit(o);
  };
  for (size_t i = 0; i < num; i++) {
    const mlb_gate_t& g = gates[i];
    const int t = g.target, c = g.control;
    auto qok = [&](int q) { return q >= 0 && (uint32_t)q < n; };
    if (g.type != 0 && !qok(t)) return fail(MLB_ERR_INVALID_QUBIT, "gate %zu: target %d", i, t);
    const bool two = (g.type >= 10 && g.type <= 13) || (g.type >= 23 && g.type <= 26);
    if ((two || g.type == MLB_GATE_ZZ) && (!qok(c) || c == t))
      return fail(MLB_ERR_INVALID_QUBIT, "gate %zu: qubits (%d,%d)", i, c, t);
    double m[8];
    switch (g.type) {
      case 0: break;                                               // I
      case 1: { mlb_op_t o{}; o.kind = MLB_OP_X; o.target = t; o.target2 = -1; emit(o); break; }
      case 2: { const double y[8] = {0, 0, 0, -1, 0, 1, 0, 0}; one(t, y); break; }   // gates.c:162
      case 3: { const double z[8] = {1, 0, 0, 0, 0, 0, -1, 0}; one(t, z); break; }   // gates.c:203
      case 4: {                                                                       // H
        const double r = 0.70710678118654752440;
        const double h[8] = {r, 0, r, 0, r, 0, -r, 0};
        one(t, h);
        break;
      }
      case 5: { const double sm[8] = {1, 0, 0, 0, 0, 0, 0, 1}; one(t, sm); break; }  // S
      case 6: mlb_mat_phase1(0, 0.0, m); one(t, m); break;                            // T
      case 7: mlb_mat_rx(g.theta, m); one(t, m); break;
      case 8: mlb_mat_ry(g.theta, m); one(t, m); break;
      case 9: mlb_mat_rz(g.theta, m); one(t, m); break;
      case 10: { mlb_op_t o{}; o.kind = MLB_OP_X; o.target = t; o.target2 = -1; o.cmask = 1ull << c; emit(o); break; }
      case 11: {  // CY composed as S . CNOT . Sdg (moonlab_qgtl_backend.c:138-144)
        const double sm[8] = {1, 0, 0, 0, 0, 0, 0, 1}, sd[8] = {1, 0, 0, 0, 0, 0, 0, -1};
        one(t, sm);
        mlb_op_t o{}; o.kind = MLB_OP_X; o.target = t; o.target2 = -1; o.cmask = 1ull << c; emit(o);
        one(t, sd);
        break;
      }
      case 12: { mlb_op_t o{}; o.kind = MLB_OP_PHASE; o.target = t; o.target2 = c; o.cmask = (1ull << t) | (1ull << c); o.m[0] = -1.0; emit(o); break; }
      case 13: { mlb_op_t o{}; o.kind = MLB_OP_SWAP; o.target = c; o.target2 = t; emit(o); break; }
      case MLB_GATE_ZZ: { mlb_op_t o{}; o.kind = MLB_OP_ZZ; o.target = c; o.target2 = t; mlb_mat_zz(g.theta, o.m); emit(o); break; }
      case 20: { const double sd[8] = {1, 0, 0, 0, 0, 0, 0, -1}; one(t, sd); break; }  // Sdg, gates.c:352
      case 21: mlb_mat_phase1(1, 0.0, m); one(t, m); break;                            // Tdg
      case 22: mlb_mat_phase1(2, g.theta, m); one(t, m); break;                        // phase(theta)
      case 23: {  // CPHASE: diag(1,1,1,e^{i theta}) (gates.c:743-754)
        mlb_op_t o{}; o.kind = MLB_OP_PHASE; o.target = t; o.target2 = c;
        o.cmask = (1ull << t) | (1ull << c); mlb_mat_cphase(g.theta, o.m); emit(o); break;
      }
      case 24: case 25: case 26: {  // CRX / CRY / CRZ GPU routes (gates.c:800-887)
        if (g.type == 24) mlb_mat_rx(g.theta, m);
        else if (g.type == 25) mlb_mat_ry(g.theta, m);
        else mlb_mat_crz_inner(g.theta, m);
        mlb_op_t o{}; o.kind = MLB_OP_1Q; o.target = t; o.target2 = -1; o.cmask = 1ull << c;
        std::memcpy(o.m, m, sizeof m); emit(o); break;
      }
      default: return fail(MLB_ERR_NOT_SUPPORTED, "gate %zu: type %d", i, g.type);
    }
  }
  *num_ops = k;
  return MLB_OK;
}

int mlb_run_gates(mlb_state_t* s, const mlb_gate_t* gates, size_t num) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  size_t cnt = 0;
  int rc = mlb_gates_to_ops(gates, num, s->n, nullptr, &cnt);
  if (rc) return rc;
  std::vector<mlb_op_t> ops(cnt);
  rc = mlb_gates_to_ops(gates, num, s->n, ops.data(), &cnt);
  if (rc) return rc;
  return mlb_apply_ops(s, ops.data(), cnt);
}

}  // extern "C"

int mlb::prepare_ops(const mlb_gate_t* gates, size_t num, uint32_t n, std::vector<mlb_op_t>& out) {
  size_t cnt = 0;
  int rc = mlb_gates_to_ops(gates, num, n, nullptr, &cnt);
  if (rc) return rc;
  std::vector<mlb_op_t> raw(cnt);
  rc = mlb_gates_to_ops(gates, num, n, raw.data(), &cnt);
  if (rc) return rc;
  mlb_state probe;  // host-side only: validation needs n
  probe.n = n;
  std::vector<mlb_op_t> q;
  q.reserve(cnt);
  for (size_t i = 0; i < cnt; i++) {
    rc = validate(&probe, raw[i]);
    if (rc) return rc;
    q.push_back(canonical(raw[i]));
  }
  out = fuse_ops(q, n);
  return MLB_OK;
}

extern "C" {

int mlb_plan_ops(const mlb_op_t* ops, size_t num, uint32_t n, int dtype, int fuse1q,
                 mlb_flush_stats_t* out) {
  if ((!ops && num) || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (n < 1 || n > 34 || (dtype != MLB_C128 && dtype != MLB_C64)) return fail(MLB_ERR_INVALID_ARG, "bad shape");
  mlb_state probe;  // host-side only: validation needs n
  probe.n = n;
  std::vector<mlb_op_t> q;
  q.reserve(num);
  for (size_t i = 0; i < num; i++) {
    int rc = validate(&probe, ops[i]);
    if (rc) return rc;
    q.push_back(canonical(ops[i]));
  }
  std::vector<mlb_op_t> fused = fuse1q ? fuse_ops(q, n) : q;
  Planner pl{n, dtype, geo(dtype)};
  pl.dense_limits = dtype == MLB_C128;  // as a state plans it by default
  pl.plan(fused);
  mlb_flush_stats_t st{};
  st.passes = pl.passes.size();
  st.segments = pl.segs.size();
  if (dtype == MLB_C128) {  // segments that run dense (the default); no matrices needed to count them
    for (const auto& pp : pl.passes)
      for (int k = 0; k < pp.pass.num_segments; k++) {
        DenseSegDev D;
        dense::SegPlan S;
        if (dense::plan_segment(pp.pass, pl.segs[pp.seg_begin + k], pl.dops.data(), D, S)) st.dense_blocks++;
      }
  }
  st.ops = fused.size();
  st.kernel_launches = pl.passes.size();
  st.bytes_moved = st.passes * 2ull * (dtype == MLB_C128 ? 16ull : 8ull) * (1ull << n);
  st.dense_amps = st.dense_blocks << n;  // a dense state: every tile of every pass
  *out = st;
  return MLB_OK;
}

int mlb_tile_plan(const mlb_op_t* ops, size_t num, uint32_t n, int dtype, int fuse1q, mlb_tile_pass_t* passes,
                  size_t* num_passes, mlb_tile_segment_t* segments, size_t* num_segments, mlb_op_t* planned,
                  size_t* num_planned) {
  if ((!ops && num) || !num_passes || !num_segments || !num_planned)
    return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (n < 1 || n > 34 || (dtype != MLB_C128 && dtype != MLB_C64)) return fail(MLB_ERR_INVALID_ARG, "bad shape");
  mlb_state probe;  // host-side only: validation needs n
  probe.n = n;
  std::vector<mlb_op_t> q;
  q.reserve(num);
  for (size_t i = 0; i < num; i++) {
    int rc = validate(&probe, ops[i]);
    if (rc) return rc;
    q.push_back(canonical(ops[i]));
  }
  const std::vector<mlb_op_t> fused = fuse1q ? fuse_ops(q, n) : q;
  Planner pl{n, dtype, geo(dtype)};
  pl.dense_limits = dtype == MLB_C128;  // as a state plans it by default
  pl.plan(fused);
  const size_t np = pl.passes.size(), ns = pl.segs.size(), no = pl.dops.size();
  const bool room = (!passes || *num_passes >= np) && (!segments || *num_segments >= ns) &&
                    (!planned || *num_planned >= no);
  *num_passes = np;
  *num_segments = ns;
  *num_planned = no;
  if (!room) return fail(MLB_ERR_INVALID_ARG, "plan buffers too small");
  for (size_t i = 0; passes && i < np; i++) {
    const PlannedPass& pp = pl.passes[i];
    mlb_tile_pass_t t{};
    t.num_low = (uint8_t)pp.pass.L;
    t.num_high = (uint8_t)pp.pass.H;
    for (int h = 0; h < pp.pass.H; h++) t.high[h] = (uint8_t)pp.pass.high[h];
    t.seg_begin = (uint32_t)pp.seg_begin;
    t.num_segments = (uint32_t)pp.pass.num_segments;
    passes[i] = t;
  }
  for (size_t i = 0; segments && i < np; i++) {
    const PlannedPass& pp = pl.passes[i];
    for (int k = pp.seg_begin; k < pp.seg_end; k++) {
      const DevSegment& sg = pl.segs[k];
      mlb_tile_segment_t t{};
      t.mode = sg.mode;
      if (dtype == MLB_C128) {
        DenseSegDev D;
        dense::SegPlan S;
        if (dense::plan_segment(pp.pass, sg, pl.dops.data(), D, S)) t.mode = 2;
      }
      t.nbits = sg.nbits;
      for (int b = 0; b < 4; b++) t.bits[b] = b < sg.nbits ? sg.bits[b] : -1;
      t.op_begin = (uint32_t)sg.op_begin;
      t.op_end = (uint32_t)sg.op_end;
      segments[k] = t;
    }
  }
  for (size_t k = 0; planned && k < no; k++) planned[k] = fused[pl.dop_src[k]];
  return MLB_OK;
}

int mlb_fused_plan(const mlb_op_t* ops, size_t num, uint32_t n, mlb_fused_pass_t* passes,
                   size_t* num_passes, mlb_fused_block_t* blocks, size_t* num_blocks, void* images,
                   size_t* image_bytes) {
  if ((!ops && num) || !num_passes || !num_blocks || !image_bytes)
    return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (n < 13 || n > 34) return fail(MLB_ERR_NOT_SUPPORTED, "the fused path needs 13..34 qubits");
  mlb_state probe;
  probe.n = n;
  std::vector<mlb_op_t> q;
  q.reserve(num);
  for (size_t i = 0; i < num; i++) {
    int rc = validate(&probe, ops[i]);
    if (rc) return rc;
    q.push_back(canonical(ops[i]));
  }
  std::vector<mlb_op_t> f1 = fuse_ops(q, n);
  fused::Plan P;
  int rc = fused::plan(f1, n, P);
  if (rc) return fail(rc, "an op spans more than 5 qubits");
  const bool fit = passes && blocks && images && *num_passes >= P.dev_passes.size() &&
                   *num_blocks >= P.dev_blocks.size() && *image_bytes >= P.images.size();
  *num_passes = P.dev_passes.size();
  *num_blocks = P.dev_blocks.size();
  *image_bytes = P.images.size();
  if (!fit) return passes || blocks || images ? fail(MLB_ERR_INVALID_ARG, "buffers too small") : MLB_OK;
  for (size_t i = 0; i < P.dev_passes.size(); i++) {
    const auto& d = P.dev_passes[i];
    std::memcpy(passes[i].hbits, d.hbits, 12);
    passes[i].num_low = d.num_low;
    passes[i].num_high = d.num_high;
    passes[i].num_tiles = d.num_tiles;
    passes[i].block_begin = d.block_begin;
    passes[i].num_blocks = d.num_blocks;
  }
  for (size_t i = 0; i < P.dev_blocks.size(); i++) {
    const auto& d = P.dev_blocks[i];
    std::memcpy(blocks[i].pos, d.pos, 5);
    std::memcpy(blocks[i].rows, d.q, 8);
    blocks[i].image = d.image;
  }
  std::memcpy(images, P.images.data(), P.images.size());
  return MLB_OK;
}

int mlb_last_flush_stats(mlb_state_t* s, mlb_flush_stats_t* out) {
  if (!s || !out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  if (s->timed_pending) {
    DeviceGuard dg(s->device);
    cudaError_t e = cudaEventSynchronize(s->t1);
    if (e != cudaSuccess) return cuda_fail(e, "timing event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->t0, s->t1);
    s->stats.gpu_ms = ms;
    s->timed_pending = false;
  }
  *out = s->stats;
  return MLB_OK;
}
int mlb_state_set_timing(mlb_state_t* s, int enable) {
  if (!s) return fail(MLB_ERR_INVALID_ARG, "null state");
  DeviceGuard dg(s->device);
  if (enable && !s->t0) {
    cudaError_t e = cudaEventCreate(&s->t0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->t1);
    if (e != cudaSuccess) return cuda_fail(e, "timing events");
  }
  s->timing = enable != 0;
  return MLB_OK;
}
int mlb_total_kernel_launches(uint64_t* out) {
  if (!out) return fail(MLB_ERR_INVALID_ARG, "null argument");
  *out = kernel_launch_count();
  return MLB_OK;
}

}  // extern "C"
