// dropin_fusion.cpp -- the reference's single-qubit gate-fusion API
// (src/optimization/fusion/fusion.h) on the engine.
//
// fuse_circuit_* / fuse_append_* keep a gate list with the reference's
// validation; fuse_compile runs the reference's run-length rule
// (fusion.c:247-292): one pending 2x2 per qubit, a 1-qubit gate multiplied in
// from the left (new = G * pending), every pending product on a qubit that a
// 2-qubit gate touches emitted as FUSED_1Q before that gate, the rest
// emitted at the end in qubit order; gate matrices as mat_of_gate builds them
// (fusion.c:41-123).  fuse_execute queues the whole list on the engine in
// one call: a GPU-backed state (quantum_state_create_gpu) runs it on its own
// device state; a host state is uploaded to a temporary device state, run,
// and read back.  The engine's tile passes then apply many gates per sweep
// of the state, where the reference dispatches one gate_* call per record.
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mlb_internal.h"
#include "moonlab_b200_dropin.h"

namespace {

using cd = std::complex<double>;

constexpr int QS_SUCCESS = 0, QS_ERROR_INVALID_STATE = -2, QS_ERROR_OUT_OF_MEMORY = -4,
              QS_ERROR_INVALID_DIMENSION = -5, QS_ERROR_NOT_SUPPORTED = -7, QS_ERROR_DRIVER = -8;
constexpr size_t kMaxQubits = 32;  // MOONLAB_MAX_QUBITS (src/quantum/state.h:44)

bool single_qubit(int k) { return k >= FUSE_GATE_H && k <= FUSE_GATE_FUSED_1Q; }

struct M2 {
  cd m[2][2];
};
M2 identity() { return {{{1.0, 0.0}, {0.0, 1.0}}}; }
M2 mul(const M2& a, const M2& b) {  // a * b
  M2 r;
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j];
  return r;
}

// The gate's 2x2 (fusion.c:41-123).
M2 matrix_of(const fuse_gate_t& g) {
  const double r2 = 0.7071067811865475244;
  const cd I(0.0, 1.0);
  M2 r = identity();
  switch (g.kind) {
    case FUSE_GATE_H: r = {{{r2, r2}, {r2, -r2}}}; break;
    case FUSE_GATE_X: r = {{{0.0, 1.0}, {1.0, 0.0}}}; break;
    case FUSE_GATE_Y: r = {{{0.0, -I}, {I, 0.0}}}; break;
    case FUSE_GATE_Z: r.m[1][1] = -1.0; break;
    case FUSE_GATE_S: r.m[1][1] = I; break;
    case FUSE_GATE_SDG: r.m[1][1] = -I; break;
    case FUSE_GATE_T: r.m[1][1] = cd(std::cos(M_PI_4), std::sin(M_PI_4)); break;
    case FUSE_GATE_TDG: r.m[1][1] = cd(std::cos(M_PI_4), -std::sin(M_PI_4)); break;
    case FUSE_GATE_PHASE: r.m[1][1] = cd(std::cos(g.p[0]), std::sin(g.p[0])); break;
    case FUSE_GATE_RX: {
      const double c = std::cos(g.p[0] / 2.0), s = std::sin(g.p[0] / 2.0);
      r = {{{c, cd(0.0, -s)}, {cd(0.0, -s), c}}};
      break;
    }
    case FUSE_GATE_RY: {
      const double c = std::cos(g.p[0] / 2.0), s = std::sin(g.p[0] / 2.0);
      r = {{{c, -s}, {s, c}}};
      break;
    }
    case FUSE_GATE_RZ: {
      const double a = g.p[0] / 2.0;
      r.m[0][0] = cd(std::cos(a), -std::sin(a));
      r.m[1][1] = cd(std::cos(a), std::sin(a));
      break;
    }
    case FUSE_GATE_U3: {
      const double th = g.p[0], ph = g.p[1], la = g.p[2];
      const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
      const cd eil(std::cos(la), std::sin(la)), eip(std::cos(ph), std::sin(ph));
      const cd eipl(std::cos(ph + la), std::sin(ph + la));
      r = {{{c, -eil * s}, {eip * s, eipl * c}}};
      break;
    }
    case FUSE_GATE_FUSED_1Q:
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) r.m[i][j] = cd(g.u[i][j][0], g.u[i][j][1]);
      break;
    default: break;
  }
  return r;
}

}  // namespace

struct fuse_circuit_t {
  size_t n = 0;
  std::vector<fuse_gate_t> gates;
};

namespace {

int push(fuse_circuit_t* c, const fuse_gate_t& g) {
  try {
    c->gates.push_back(g);
  } catch (...) {
    return -1;
  }
  return 0;
}
int add1(fuse_circuit_t* c, int kind, int q, double p0) {
  if (!c || q < 0 || (size_t)q >= c->n) return -1;
  fuse_gate_t g{};
  g.kind = kind;
  g.q[0] = q;
  g.q[1] = -1;
  g.p[0] = p0;
  return push(c, g);
}
int add2(fuse_circuit_t* c, int kind, int a, int b, double p0) {
  if (!c || a < 0 || (size_t)a >= c->n || b < 0 || (size_t)b >= c->n || a == b) return -1;
  fuse_gate_t g{};
  g.kind = kind;
  g.q[0] = a;
  g.q[1] = b;
  g.p[0] = p0;
  return push(c, g);
}

// One fuse record as engine ops (appended to out); false if unknown.
bool to_ops(const fuse_gate_t& g, uint32_t n, std::vector<mlb_op_t>& out) {
  if (g.kind == FUSE_GATE_FUSED_1Q || g.kind == FUSE_GATE_U3 || g.kind == FUSE_GATE_CY) {
    // CY is gate_cy's controlled Y (gates.c:670-697), not the QGTL record's
    // S . CNOT . Sdg composition
    const M2 m = g.kind == FUSE_GATE_CY ? M2{{{0.0, cd(0.0, -1.0)}, {cd(0.0, 1.0), 0.0}}} : matrix_of(g);
    mlb_op_t o{};
    o.kind = MLB_OP_1Q;
    o.target = g.kind == FUSE_GATE_CY ? g.q[1] : g.q[0];
    o.target2 = -1;
    if (g.kind == FUSE_GATE_CY) o.cmask = 1ull << g.q[0];
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        o.m[2 * (2 * i + j)] = m.m[i][j].real();
        o.m[2 * (2 * i + j) + 1] = m.m[i][j].imag();
      }
    out.push_back(o);
    return true;
  }
  // gate records (QGTL numbering and its extensions, include/moonlab_b200.h)
  static const int type_of[] = {4, 1, 2, 3, 5, 20, 6, 21, 22, 7, 8, 9, -1, -1, 10, 12, -1, 13, 23, 24, 25, 26};
  if (g.kind < 0 || g.kind > FUSE_GATE_CRZ || type_of[g.kind] < 0) return false;
  mlb_gate_t rec{};
  rec.type = type_of[g.kind];
  rec.theta = g.p[0];
  if (single_qubit(g.kind)) {
    rec.target = g.q[0];
    rec.control = -1;
  } else {  // q[0] = control (the first qubit of SWAP), q[1] = target
    rec.control = g.q[0];
    rec.target = g.q[1];
  }
  size_t cnt = 0;
  if (mlb_gates_to_ops(&rec, 1, n, nullptr, &cnt) != MLB_OK) return false;
  const size_t at = out.size();
  out.resize(at + cnt);
  return mlb_gates_to_ops(&rec, 1, n, out.data() + at, &cnt) == MLB_OK;
}

}  // namespace

extern "C" {

fuse_circuit_t* fuse_circuit_create(size_t num_qubits) {
  if (num_qubits == 0 || num_qubits > kMaxQubits) return nullptr;
  auto* c = new (std::nothrow) fuse_circuit_t();
  if (!c) return nullptr;
  c->n = num_qubits;
  c->gates.reserve(16);
  return c;
}
void fuse_circuit_free(fuse_circuit_t* c) { delete c; }
size_t fuse_circuit_len(const fuse_circuit_t* c) { return c ? c->gates.size() : 0; }
size_t fuse_circuit_num_qubits(const fuse_circuit_t* c) { return c ? c->n : 0; }

int fuse_append_h(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_H, q, 0); }
int fuse_append_x(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_X, q, 0); }
int fuse_append_y(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_Y, q, 0); }
int fuse_append_z(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_Z, q, 0); }
int fuse_append_s(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_S, q, 0); }
int fuse_append_sdg(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_SDG, q, 0); }
int fuse_append_t(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_T, q, 0); }
int fuse_append_tdg(fuse_circuit_t* c, int q) { return add1(c, FUSE_GATE_TDG, q, 0); }
int fuse_append_phase(fuse_circuit_t* c, int q, double t) { return add1(c, FUSE_GATE_PHASE, q, t); }
int fuse_append_rx(fuse_circuit_t* c, int q, double t) { return add1(c, FUSE_GATE_RX, q, t); }
int fuse_append_ry(fuse_circuit_t* c, int q, double t) { return add1(c, FUSE_GATE_RY, q, t); }
int fuse_append_rz(fuse_circuit_t* c, int q, double t) { return add1(c, FUSE_GATE_RZ, q, t); }
int fuse_append_u3(fuse_circuit_t* c, int q, double theta, double phi, double lambda) {
  if (add1(c, FUSE_GATE_U3, q, theta)) return -1;
  c->gates.back().p[1] = phi;
  c->gates.back().p[2] = lambda;
  return 0;
}
int fuse_append_cnot(fuse_circuit_t* c, int a, int b) { return add2(c, FUSE_GATE_CNOT, a, b, 0); }
int fuse_append_cz(fuse_circuit_t* c, int a, int b) { return add2(c, FUSE_GATE_CZ, a, b, 0); }
int fuse_append_cy(fuse_circuit_t* c, int a, int b) { return add2(c, FUSE_GATE_CY, a, b, 0); }
int fuse_append_swap(fuse_circuit_t* c, int a, int b) { return add2(c, FUSE_GATE_SWAP, a, b, 0); }
int fuse_append_cphase(fuse_circuit_t* c, int a, int b, double t) { return add2(c, FUSE_GATE_CPHASE, a, b, t); }
int fuse_append_crx(fuse_circuit_t* c, int a, int b, double t) { return add2(c, FUSE_GATE_CRX, a, b, t); }
int fuse_append_cry(fuse_circuit_t* c, int a, int b, double t) { return add2(c, FUSE_GATE_CRY, a, b, t); }
int fuse_append_crz(fuse_circuit_t* c, int a, int b, double t) { return add2(c, FUSE_GATE_CRZ, a, b, t); }

fuse_circuit_t* fuse_compile(const fuse_circuit_t* src, fuse_stats_t* stats) {
  if (!src) return nullptr;
  fuse_circuit_t* dst = fuse_circuit_create(src->n);
  if (!dst) return nullptr;
  if (stats) {
    stats->original_gates = src->gates.size();
    stats->fused_gates = 0;
    stats->merges_applied = 0;
  }
  struct Pending {
    M2 m;
    int count = 0;
  };
  std::vector<Pending> pend(src->n);
  auto flush = [&](int q) {
    Pending& p = pend[q];
    if (!p.count) return 0;
    fuse_gate_t g{};
    g.kind = FUSE_GATE_FUSED_1Q;
    g.q[0] = q;
    g.q[1] = -1;
    for (int i = 0; i < 2; i++)
      for (int j = 0; j < 2; j++) {
        g.u[i][j][0] = p.m.m[i][j].real();
        g.u[i][j][1] = p.m.m[i][j].imag();
      }
    if (stats) stats->merges_applied += (size_t)(p.count - 1);
    p.count = 0;
    return push(dst, g);
  };
  for (const fuse_gate_t& g : src->gates) {
    int rc = 0;
    if (single_qubit(g.kind)) {
      Pending& p = pend[g.q[0]];
      const M2 gm = matrix_of(g);
      p.m = p.count ? mul(gm, p.m) : gm;  // applied after what is pending
      p.count++;
    } else {
      rc = flush(g.q[0]);
      if (!rc) rc = flush(g.q[1]);
      if (!rc) rc = push(dst, g);
    }
    if (rc) {
      fuse_circuit_free(dst);
      return nullptr;
    }
  }
  for (size_t q = 0; q < src->n; q++)
    if (flush((int)q)) {
      fuse_circuit_free(dst);
      return nullptr;
    }
  if (stats) stats->fused_gates = dst->gates.size();
  return dst;
}

int mlb_fuse_circuit_ops(const fuse_circuit_t* c, uint32_t num_qubits, void* ops, size_t capacity,
                         size_t* num_ops) {
  if (!c || !num_ops) return MLB_ERR_INVALID_ARG;
  if (num_qubits < c->n) return MLB_ERR_NUM_QUBITS;
  std::vector<mlb_op_t> v;
  for (const fuse_gate_t& g : c->gates)
    if (!to_ops(g, num_qubits, v)) return MLB_ERR_INVALID_ARG;
  *num_ops = v.size();
  if (ops) {
    if (capacity < v.size()) return MLB_ERR_INVALID_ARG;
    std::memcpy(ops, v.data(), v.size() * sizeof(mlb_op_t));
  }
  return MLB_OK;
}

qs_error_t fuse_execute(const fuse_circuit_t* c, quantum_state_t* state) {
  if (!c || !state) return QS_ERROR_INVALID_STATE;
  if (state->num_qubits < c->n) return QS_ERROR_INVALID_DIMENSION;
  const uint32_t n = (uint32_t)state->num_qubits;
  std::vector<mlb_op_t> ops;
  ops.reserve(c->gates.size());
  for (const fuse_gate_t& g : c->gates)
    if (!to_ops(g, n, ops)) return QS_ERROR_INVALID_STATE;
  mlb_state_t* e = moonlab_b200_engine_of(state);
  if (e) return mlb_apply_ops(e, ops.data(), ops.size()) == MLB_OK ? QS_SUCCESS : QS_ERROR_DRIVER;
  // a host state: run it on a temporary device state
  if (!state->amplitudes) return QS_ERROR_INVALID_STATE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return QS_ERROR_NOT_SUPPORTED;
  }
  mlb_state_t* t = nullptr;
  int rc = mlb_state_create(n, MLB_C128, dev, &t);
  if (rc != MLB_OK) return rc == MLB_ERR_OUT_OF_MEMORY ? QS_ERROR_OUT_OF_MEMORY : QS_ERROR_NOT_SUPPORTED;
  rc = mlb_state_copy_from_host(t, state->amplitudes);
  if (rc == MLB_OK) rc = mlb_apply_ops(t, ops.data(), ops.size());
  if (rc == MLB_OK) rc = mlb_state_copy_to_host(t, state->amplitudes);
  mlb_state_free(t);
  return rc == MLB_OK ? QS_SUCCESS : QS_ERROR_DRIVER;
}

}  // extern "C"
