// dropin_vqe.cpp -- moonlab_vqe_gradient on the batched adjoint engine.
//
// Reads the reference's public solver layout (src/algorithms/vqe.h) and
// mirrors its exact-or-error contract (vqe.c:2033-2070 via
// moonlab_vqe_export.c:27-42).  Hamiltonians are cached by content so a
// solver loop re-plans nothing.
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

int gradient(void* solver_v, size_t batch, const double* params, double* grads, size_t P) {
  if (!solver_v || !params || !grads) return -1;
  auto* s = static_cast<vqe_solver_t*>(solver_v);
  if (!s->ansatz || s->ansatz->num_parameters != P) return -2;
  if (!s->hamiltonian) return -3;
  if (s->noise_model && s->noise_model->enabled) return -3;  // no exact gradient under noise
  if (s->ansatz->type != 0) return -3;                       // adjoint tape is the HEA one
  if (s->ansatz->num_parameters != 2 * s->ansatz->num_qubits * s->ansatz->num_layers) return -3;
  std::lock_guard<std::mutex> lk(g_mu);
  mlb_hea_t* h = lookup(s);
  if (!h) return -3;
  return mlb_hea_evaluate(h, batch, params, nullptr, grads, 0) == MLB_OK ? 0 : -3;
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

}  // extern "C"
