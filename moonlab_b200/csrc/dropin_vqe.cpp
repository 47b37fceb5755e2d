// dropin_vqe.cpp -- the reference's stable VQE verbs on the engine:
// moonlab_vqe_gradient, moonlab_vqe_qgt, moonlab_vqe_berry_curvature and
// moonlab_vqe_natural_gradient (src/applications/moonlab_vqe_export.c).
//
// Reads the reference's public solver layout (src/algorithms/vqe.h) and
// mirrors each verb's contract (0 ok, -1 NULL, -2 parameter count, -3
// failure).  Hardware-efficient ansatz: the batched adjoint engine
// (gradient) and its batched derivative states + FP64 Gram kernel
// (geometry).  UCCSD and symmetry-preserving ansatz, noise-free: the
// reference's exact parameter-shift rules (vqe.c:2072-2140), every shifted
// energy a circuit run and a Pauli-sum reduction on the device.  What the
// engine does not model -- a CUSTOM ansatz (a host callback) and a noisy
// solver that opted into stochastic parameter shift -- is handed to the
// reference's own vqe_compute_gradient / vqe_compute_qgt /
// vqe_compute_berry_curvature / vqe_natural_gradient_direction when the
// process has them (the reference core library), else -3.  Hamiltonians
// are cached by content so a solver loop re-plans nothing.
#include <dlfcn.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "mlb_internal.h"
#include "moonlab_b200_dropin.h"

namespace {

// src/algorithms/vqe.h:101-127, 232-241, 545-568; src/quantum/noise.h:86-106
struct pauli_term_t {
  double coefficient;
  char* pauli_string;
  size_t num_qubits;
};
struct pauli_hamiltonian_t {
  size_t num_qubits;
  size_t num_terms;
  pauli_term_t* terms;
  double nuclear_repulsion;
  char* molecule_name;
  double bond_distance;
  uint64_t hf_reference;
};
struct vqe_ansatz_t {
  int type;  // vqe_ansatz_type_t; 0 = VQE_ANSATZ_HARDWARE_EFFICIENT
  size_t num_qubits;
  size_t num_layers;
  size_t num_parameters;
  double* parameters;
  void* circuit_data;
};
struct noise_model_head_t {
  int enabled;
};
struct vqe_solver_t {
  pauli_hamiltonian_t* hamiltonian;
  vqe_ansatz_t* ansatz;
  void* optimizer;
  void* entropy;
  noise_model_head_t* noise_model;
  size_t iteration;
  double* energy_history;
  size_t max_history;
  size_t total_measurements;
  double total_time;
  int allow_stochastic_gradient;
};
enum { ANSATZ_HEA = 0, ANSATZ_UCCSD = 1, ANSATZ_CUSTOM = 2, ANSATZ_SYMMETRY = 3 };  // vqe.h:219-224
struct uccsd_data_t {  // vqe.c:586-591
  size_t num_occupied, num_virtual, num_singles, num_doubles;
};
struct sym_preserve_data_t {  // vqe.c:603-606
  size_t num_occupied, num_virtual;
};

struct Entry {
  std::vector<unsigned char> key;
  mlb_hea_t* h = nullptr;
};
std::mutex g_mu;
std::vector<Entry> g_cache;

// Convert the Pauli strings (char per qubit, index = qubit, I/X/Y/Z either
// case, vqe.c:1889-1941) into X/Z masks; -1 on an invalid character.
int masks_of(const pauli_hamiltonian_t* H, size_t n, std::vector<uint64_t>& xm, std::vector<uint64_t>& zm,
             std::vector<double>& c) {
  for (size_t k = 0; k < H->num_terms; k++) {
    const pauli_term_t& t = H->terms[k];
    uint64_t x = 0, z = 0;
    if (t.pauli_string) {
      for (size_t q = 0; q < t.num_qubits; q++) {
        const char ch = t.pauli_string[q];
        if (ch == 'I' || ch == 'i') continue;
        if (q >= n) return -1;
        if (ch == 'X' || ch == 'x') x |= 1ull << q;
        else if (ch == 'Y' || ch == 'y') { x |= 1ull << q; z |= 1ull << q; }
        else if (ch == 'Z' || ch == 'z') z |= 1ull << q;
        else return -1;
      }
    }
    xm.push_back(x);
    zm.push_back(z);
    c.push_back(t.coefficient);
  }
  return 0;
}

mlb_hea_t* lookup(const vqe_solver_t* s) {
  const pauli_hamiltonian_t* H = s->hamiltonian;
  const vqe_ansatz_t* A = s->ansatz;
  std::vector<uint64_t> xm, zm;
  std::vector<double> c;
  if (masks_of(H, A->num_qubits, xm, zm, c)) return nullptr;
  std::vector<unsigned char> key;
  auto put = [&](const void* p, size_t b) {
    const unsigned char* q = (const unsigned char*)p;
    key.insert(key.end(), q, q + b);
  };
  const uint64_t shape[3] = {A->num_qubits, A->num_layers, H->hf_reference};
  put(shape, sizeof shape);
  put(xm.data(), xm.size() * 8);
  put(zm.data(), zm.size() * 8);
  put(c.data(), c.size() * 8);
  for (auto& e : g_cache)
    if (e.key == key) return e.h;
  int dev = 0;
  cudaGetDevice(&dev);
  mlb_hea_t* h = nullptr;
  if (mlb_hea_create((uint32_t)A->num_qubits, (uint32_t)A->num_layers, H->hf_reference, xm.size(), xm.data(),
                     zm.data(), c.data(), MLB_C128, dev, &h) != MLB_OK)
    return nullptr;
  if (g_cache.size() >= 8) {
    mlb_hea_free(g_cache.front().h);
    g_cache.erase(g_cache.begin());
  }
  g_cache.push_back({std::move(key), h});
  return h;
}

bool noisy(const vqe_solver_t* s) { return s->noise_model && s->noise_model->enabled; }

bool is_hea(const vqe_solver_t* s) {
  return s->ansatz->type == ANSATZ_HEA &&
         s->ansatz->num_parameters == 2 * s->ansatz->num_qubits * s->ansatz->num_layers;
}

// The reference's own entry for what the engine does not model, when the
// process has the reference core (resolved at run time; no link dependency).
template <typename F>
F reference_fn(const char* name) {
  return reinterpret_cast<F>(dlsym(RTLD_DEFAULT, name));
}

extern "C" void mlb_mat_ry(double theta, double m[8]);

// Engine ops of the noise-free ansatz on |hf>: the X prefix (vqe_compute_energy,
// vqe.c:1298-1301), then vqe_apply_uccsd_ansatz (vqe.c:786-845) or
// vqe_apply_symmetry_preserving_ansatz (vqe.c:700-723).
void op_x(std::vector<mlb_op_t>& ops, int t, uint64_t cmask) {
  mlb_op_t o{};
  o.kind = MLB_OP_X;
  o.target = t;
  o.target2 = -1;
  o.cmask = cmask;
  ops.push_back(o);
}
// gate_cry (gates.c:833-846): RY(theta) on target where the control is 1
void op_cry(std::vector<mlb_op_t>& ops, int c, int t, double theta) {
  mlb_op_t o{};
  o.kind = MLB_OP_1Q;
  o.target = t;
  o.target2 = -1;
  o.cmask = 1ull << c;
  mlb_mat_ry(theta, o.m);
  ops.push_back(o);
}
// vqe_apply_givens_rotation (vqe.c:847-878): CNOT(a, i) CRY(i -> a) CNOT(a, i)
void op_givens(std::vector<mlb_op_t>& ops, int i, int a, double theta) {
  op_x(ops, i, 1ull << a);
  op_cry(ops, i, a, theta);
  op_x(ops, i, 1ull << a);
}
// vqe_apply_double_excitation (vqe.c:880-941): the rotation
// |1_i 1_j 0_a 0_b> -> c |1100> + s |0011>, |0011> -> -s |1100> + c |0011>
// (c = cos theta, s = sin theta), identity elsewhere.  CNOTs from i onto j,
// a and b map the pair to two states that differ only in bit i, with j = 0
// and a = b = 1; there it is one 2x2 rotation on i controlled by (not j), a
// and b ([[c, s], [-s, c]] on (i = 0, i = 1)), and the CNOTs are undone.
void op_double(std::vector<mlb_op_t>& ops, int i, int j, int a, int b, double theta) {
  const int tg[3] = {j, a, b};
  for (int t : tg) op_x(ops, t, 1ull << i);
  op_x(ops, j, 0);
  mlb_op_t o{};
  o.kind = MLB_OP_1Q;
  o.target = i;
  o.target2 = -1;
  o.cmask = (1ull << j) | (1ull << a) | (1ull << b);
  const double c = std::cos(theta), sn = std::sin(theta);
  o.m[0] = c;
  o.m[2] = sn;
  o.m[4] = -sn;
  o.m[6] = c;
  ops.push_back(o);
  op_x(ops, j, 0);
  for (int k = 2; k >= 0; k--) op_x(ops, tg[k], 1ull << i);
}

bool ansatz_ops(const vqe_solver_t* s, const double* theta, std::vector<mlb_op_t>& ops) {
  const vqe_ansatz_t* A = s->ansatz;
  const size_t n = A->num_qubits;
  ops.clear();
  for (size_t q = 0; q < n; q++)
    if (s->hamiltonian->hf_reference >> q & 1ull) op_x(ops, (int)q, 0);
  size_t p = 0;
  if (A->type == ANSATZ_UCCSD) {
    const auto* d = static_cast<const uccsd_data_t*>(A->circuit_data);
    if (!d) return false;
    for (size_t i = 0; i < d->num_occupied; i++)
      for (size_t a = 0; a < d->num_virtual; a++) op_givens(ops, (int)i, (int)(d->num_occupied + a), theta[p++]);
    for (size_t i = 0; i < d->num_occupied; i++)
      for (size_t j = i + 1; j < d->num_occupied; j++)
        for (size_t a = 0; a < d->num_virtual; a++)
          for (size_t b = a + 1; b < d->num_virtual; b++)
            op_double(ops, (int)i, (int)j, (int)(d->num_occupied + a), (int)(d->num_occupied + b), theta[p++]);
  } else if (A->type == ANSATZ_SYMMETRY) {
    const auto* d = static_cast<const sym_preserve_data_t*>(A->circuit_data);
    if (!d) return false;
    for (size_t l = 0; l < A->num_layers; l++)
      for (size_t o = 0; o < d->num_occupied; o++)
        for (size_t v = 0; v < d->num_virtual; v++) {
          const int qo = (int)(d->num_virtual + o), qv = (int)v;
          op_x(ops, qo, 1ull << qv);
          op_cry(ops, qo, qv, theta[p++]);
          op_x(ops, qo, 1ull << qv);
        }
  } else {
    return false;
  }
  return p == A->num_parameters;
}

// Noise-free parameter shift for the excitation ansaetze (vqe.c:2072-2140):
// the four-term rule c1 [E(+pi/2) - E(-pi/2)] + c2 [E(+3pi/2) - E(-3pi/2)]
// for generators with spectrum {-1/2, 0, 1/2}.  Every energy is the ansatz
// on one engine state and a device Pauli-sum reduction; the shifted
// circuits share one shape, so the state's plan cache replays them.
int psr_gradient(vqe_solver_t* s, const double* params, double* grad) {
  const size_t P = s->ansatz->num_parameters, n = s->ansatz->num_qubits;
  std::vector<uint64_t> xm, zm;
  std::vector<double> c;
  if (masks_of(s->hamiltonian, n, xm, zm, c)) return -3;
  int dev = 0;
  cudaGetDevice(&dev);
  mlb_state_t* st = nullptr;
  if (mlb_state_create((uint32_t)n, MLB_C128, dev, &st) != MLB_OK) return -3;
  mlb_state_set_plan_cache(st, 4);
  std::vector<double> base(params, params + P), th(base);
  std::vector<mlb_op_t> ops;
  int rc = 0;
  auto energy = [&](double& e) {
    if (!ansatz_ops(s, th.data(), ops)) return false;
    if (mlb_state_reset(st) != MLB_OK || mlb_apply_ops(st, ops.data(), ops.size()) != MLB_OK) return false;
    if (mlb_expect_pauli_sum(st, xm.size(), xm.data(), zm.data(), c.data(), &e) != MLB_OK) return false;
    e += s->hamiltonian->nuclear_repulsion;
    s->total_measurements += xm.size();
    return true;
  };
  const double c1 = 0.25 + M_SQRT2 / 8.0, c2 = M_SQRT2 / 8.0 - 0.25;
  for (size_t i = 0; i < P && rc == 0; i++) {
    double ep1, em1, ep3, em3;
    th[i] = base[i] + M_PI / 2.0;
    bool ok = energy(ep1);
    th[i] = base[i] - M_PI / 2.0;
    ok = ok && energy(em1);
    th[i] = base[i] + 3.0 * M_PI / 2.0;
    ok = ok && energy(ep3);
    th[i] = base[i] - 3.0 * M_PI / 2.0;
    ok = ok && energy(em3);
    th[i] = base[i];
    if (!ok) rc = -3;
    else grad[i] = c1 * (ep1 - em1) + c2 * (ep3 - em3);
  }
  mlb_state_free(st);
  if (rc == 0) std::memcpy(s->ansatz->parameters, base.data(), P * sizeof(double));
  return rc;
}

int gradient(void* solver_v, size_t batch, const double* params, double* grads, size_t P) {
  if (!solver_v || !params || !grads) return -1;
  auto* s = static_cast<vqe_solver_t*>(solver_v);
  if (!s->ansatz || s->ansatz->num_parameters != P) return -2;
  if (!s->hamiltonian) return -3;
  if (noisy(s) || !is_hea(s)) {
    // exact-or-error: a noisy solver gets no gradient unless it opted into
    // stochastic parameter shift (vqe.c:2060-2066)
    if (noisy(s) && !s->allow_stochastic_gradient) return -3;
    if (!noisy(s) && (s->ansatz->type == ANSATZ_UCCSD || s->ansatz->type == ANSATZ_SYMMETRY)) {
      std::lock_guard<std::mutex> lk(g_mu);
      for (size_t b = 0; b < batch; b++)
        if (int rc = psr_gradient(s, params + b * P, grads + b * P)) return rc;
      return 0;
    }
    using Fn = int (*)(void*, const double*, double*);
    Fn f = reference_fn<Fn>("vqe_compute_gradient");
    if (!f) return -3;
    for (size_t b = 0; b < batch; b++)
      if (f(s, params + b * P, grads + b * P) != 0) return -3;
    return 0;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  mlb_hea_t* h = lookup(s);
  if (!h) return -3;
  return mlb_hea_evaluate(h, batch, params, nullptr, grads, 0) == MLB_OK ? 0 : -3;
}

// Gaussian elimination with partial pivoting on (g + reg I) x = grad, as
// spd_solve does it (vqe_qng.c:236-266): singular (pivot below 1e-300) -> -1.
int spd_solve(std::vector<double>& A, const double* b, double* x, size_t n) {
  std::vector<double> w(b, b + n);
  for (size_t col = 0; col < n; col++) {
    size_t piv = col;
    double best = std::fabs(A[col * n + col]);
    for (size_t r = col + 1; r < n; r++) {
      const double v = std::fabs(A[r * n + col]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (best < 1e-300) return -1;
    if (piv != col) {
      for (size_t k = 0; k < n; k++) std::swap(A[col * n + k], A[piv * n + k]);
      std::swap(w[col], w[piv]);
    }
    const double diag = A[col * n + col];
    for (size_t r = col + 1; r < n; r++) {
      const double f = A[r * n + col] / diag;
      if (f == 0.0) continue;
      for (size_t k = col; k < n; k++) A[r * n + k] -= f * A[col * n + k];
      w[r] -= f * w[col];
    }
  }
  for (size_t ii = n; ii-- > 0;) {
    double acc = w[ii];
    for (size_t k = ii + 1; k < n; k++) acc -= A[ii * n + k] * x[k];
    x[ii] = acc / A[ii * n + ii];
  }
  return 0;
}

// Geometry verbs: common argument checks (moonlab_vqe_export.c:53-100).
int geo_check(void* solver_v, const void* a, const void* b, size_t P) {
  if (!solver_v || !a || !b) return -1;
  auto* s = static_cast<vqe_solver_t*>(solver_v);
  if (!s->ansatz || s->ansatz->num_parameters != P) return -2;
  if (!s->hamiltonian) return -3;
  return 0;
}

int hea_geometry(vqe_solver_t* s, const double* params, double* metric, double* curvature) {
  std::lock_guard<std::mutex> lk(g_mu);
  mlb_hea_t* h = lookup(s);
  if (!h) return -3;
  return mlb_hea_geometry(h, params, metric, curvature) == MLB_OK ? 0 : -3;
}

}  // namespace

extern "C" {

int moonlab_vqe_gradient(void* solver, const double* parameters, double* gradient_out, size_t num_parameters) {
  return gradient(solver, 1, parameters, gradient_out, num_parameters);
}

int moonlab_b200_vqe_gradient_batch(void* solver, size_t batch, const double* parameters, double* gradients_out,
                                    size_t num_parameters) {
  if (batch == 0) return solver && parameters && gradients_out ? 0 : -1;
  return gradient(solver, batch, parameters, gradients_out, num_parameters);
}

int moonlab_vqe_qgt(void* solver, const double* parameters, double* qgt_out, size_t num_parameters) {
  if (int rc = geo_check(solver, parameters, qgt_out, num_parameters)) return rc;
  auto* s = static_cast<vqe_solver_t*>(solver);
  if (is_hea(s)) return hea_geometry(s, parameters, qgt_out, nullptr);
  using Fn = int (*)(void*, const double*, double*);
  Fn f = reference_fn<Fn>("vqe_compute_qgt");
  return f && f(s, parameters, qgt_out) == 0 ? 0 : -3;
}

int moonlab_vqe_berry_curvature(void* solver, const double* parameters, double* berry_out,
                                size_t num_parameters) {
  if (int rc = geo_check(solver, parameters, berry_out, num_parameters)) return rc;
  auto* s = static_cast<vqe_solver_t*>(solver);
  if (is_hea(s)) return hea_geometry(s, parameters, nullptr, berry_out);
  using Fn = int (*)(void*, const double*, double*);
  Fn f = reference_fn<Fn>("vqe_compute_berry_curvature");
  return f && f(s, parameters, berry_out) == 0 ? 0 : -3;
}

int moonlab_vqe_natural_gradient(void* solver, const double* parameters, const double* gradient,
                                 double regularization, double* direction_out, size_t num_parameters) {
  if (!gradient) return -1;
  if (int rc = geo_check(solver, parameters, direction_out, num_parameters)) return rc;
  auto* s = static_cast<vqe_solver_t*>(solver);
  if (!is_hea(s)) {
    using Fn = int (*)(void*, const double*, const double*, double, double*);
    Fn f = reference_fn<Fn>("vqe_natural_gradient_direction");
    return f && f(s, parameters, gradient, regularization, direction_out) == 0 ? 0 : -3;
  }
  const size_t P = num_parameters;
  std::vector<double> g(P * P);
  if (hea_geometry(s, parameters, g.data(), nullptr) != 0) return -3;
  for (size_t i = 0; i < P; i++) g[i * P + i] += regularization;  // Tikhonov (vqe_qng.c:279)
  return spd_solve(g, gradient, direction_out, P) == 0 ? 0 : -3;
}

}  // extern "C"
