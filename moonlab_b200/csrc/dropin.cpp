// dropin.cpp -- strong definitions of the reference's GPU-backend symbols,
// implemented on the B200 engine (see include/moonlab_b200_dropin.h for the
// reference interface each one replaces).
#include <cstdlib>
#include <cstring>

#include "mlb_internal.h"
#include "moonlab_b200_dropin.h"

namespace {

// QS_* (src/quantum/state.h:78-88)
constexpr int QS_SUCCESS = 0, QS_ERROR_OUT_OF_MEMORY = -4, QS_ERROR_INVALID_PARAM = -6,
              QS_ERROR_NOT_SUPPORTED = -7, QS_ERROR_DRIVER = -8;

mlb_state* eng(quantum_state_t* s) {
  return (s && s->gpu_state) ? static_cast<mlb_state*>(s->gpu_state) : nullptr;
}
int route(int rc) { return rc == MLB_OK ? 0 : -1; }

}  // namespace

extern "C" {

// ---- GPU-backed quantum_state_t ----------------------------------------------
// state_gpu.cu:31-72: calloc'ed host mirror holding |0...0>, opaque engine
// state in gpu_state, gpu_backend = 1.  The mirror cannot be left out until
// the first sync: the core's gate functions refuse a state whose amplitudes
// pointer is NULL before they route to the device (gates.c:124, :157, ...).
// calloc maps a block this large on demand, so the mirror's pages take host
// memory only once sync_to_host writes them (the page holding amplitude 0
// aside).  Errors: no device -> NOT_SUPPORTED, allocation failure ->
// OUT_OF_MEMORY.
qs_error_t quantum_state_create_gpu(size_t num_qubits, quantum_state_t** out_state) {
  if (!out_state) return QS_ERROR_INVALID_PARAM;
  *out_state = nullptr;
  if (num_qubits == 0 || num_qubits > 33) return QS_ERROR_INVALID_PARAM;
  auto* s = static_cast<quantum_state_t*>(calloc(1, sizeof(quantum_state_t)));
  if (!s) return QS_ERROR_OUT_OF_MEMORY;
  s->num_qubits = num_qubits;
  s->state_dim = (size_t)1 << num_qubits;
  s->amplitudes = calloc(s->state_dim, 2 * sizeof(double));
  if (!s->amplitudes) {
    free(s);
    return QS_ERROR_OUT_OF_MEMORY;
  }
  static_cast<double*>(s->amplitudes)[0] = 1.0;
  s->owns_memory = 1;
  int dev = 0;
  cudaGetDevice(&dev);
  mlb_state* e = nullptr;
  const int rc = mlb_state_create((uint32_t)num_qubits, MLB_C128, dev, &e);
  if (rc != MLB_OK) {
    free(s->amplitudes);
    free(s);
    return (rc == MLB_ERR_NO_DEVICE || rc == MLB_ERR_DRIVER) ? QS_ERROR_NOT_SUPPORTED : QS_ERROR_OUT_OF_MEMORY;
  }
  s->gpu_state = e;
  s->gpu_backend = 1;
  *out_state = s;
  return QS_SUCCESS;
}

// state_gpu.cu:74-86
qs_error_t quantum_state_sync_to_host(quantum_state_t* state) {
  if (!state) return QS_ERROR_INVALID_PARAM;
  mlb_state* e = eng(state);
  if (!e) return QS_SUCCESS;
  return mlb_state_copy_to_host(e, state->amplitudes) == MLB_OK ? QS_SUCCESS : QS_ERROR_DRIVER;
}

// state_gpu.cu:88-98
qs_error_t quantum_state_sync_from_host(quantum_state_t* state) {
  if (!state) return QS_ERROR_INVALID_PARAM;
  mlb_state* e = eng(state);
  if (!e) return QS_SUCCESS;
  return mlb_state_copy_from_host(e, state->amplitudes) == MLB_OK ? QS_SUCCESS : QS_ERROR_DRIVER;
}

mlb_state* moonlab_b200_engine_of(quantum_state_t* state) { return eng(state); }

// ---- routing (state_gpu.cu:108-199) ---------------------------------------
int qsim_gpu_route_cnot(quantum_state_t* s, int control, int target) {
  mlb_state* e = eng(s);
  if (!e || control < 0 || target < 0 || control >= 64) return -1;
  return route(mlb_apply_mcx(e, 1ull << control, (uint32_t)target));
}
int qsim_gpu_route_hadamard(quantum_state_t* s, int qubit) {
  mlb_state* e = eng(s);
  if (!e || qubit < 0) return -1;
  return route(moonlab_cuda_apply_h(e, (uint32_t)qubit));
}
int qsim_gpu_route_pauli_x(quantum_state_t* s, int qubit) {
  mlb_state* e = eng(s);
  if (!e || qubit < 0) return -1;
  return route(mlb_apply_mcx(e, 0, (uint32_t)qubit));
}
int qsim_gpu_route_apply_1q_matrix(quantum_state_t* s, int qubit, const double m[8]) {
  mlb_state* e = eng(s);
  if (!e || !m || qubit < 0) return -1;
  return route(mlb_apply_1q(e, (uint32_t)qubit, m));
}
int qsim_gpu_route_apply_2q_matrix(quantum_state_t* s, int q0, int q1, const double m[32]) {
  mlb_state* e = eng(s);
  if (!e || !m || q0 < 0 || q1 < 0) return -1;
  return route(mlb_apply_2q(e, (uint32_t)q0, (uint32_t)q1, m));
}
int qsim_gpu_route_mcx(quantum_state_t* s, uint64_t control_mask, int target) {
  mlb_state* e = eng(s);
  if (!e || target < 0) return -1;
  return route(mlb_apply_mcx(e, control_mask, (uint32_t)target));
}
int qsim_gpu_route_mcz(quantum_state_t* s, uint64_t all_mask) {
  mlb_state* e = eng(s);
  if (!e || all_mask == 0) return -1;
  return route(mlb_apply_mcz(e, all_mask));
}
int qsim_gpu_route_fredkin(quantum_state_t* s, int control, int t1, int t2) {
  mlb_state* e = eng(s);
  if (!e || control < 0 || control >= 64 || t1 < 0 || t2 < 0) return -1;
  return route(mlb_apply_swap(e, 1ull << control, (uint32_t)t1, (uint32_t)t2));
}

// ---- moonlab_cuda_* (cuda_statevec.h) --------------------------------------
moonlab_cuda_status_t moonlab_cuda_state_create(uint32_t n_qubits, moonlab_cuda_state_t** out) {
  if (!out) return MLB_ERR_INVALID_ARG;
  if (n_qubits < 1 || n_qubits > 33) return MLB_ERR_NUM_QUBITS;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return MLB_ERR_NO_DEVICE;
  }
  return mlb_state_create(n_qubits, MLB_C128, dev, out);
}
void moonlab_cuda_state_free(moonlab_cuda_state_t* s) { mlb_state_free(s); }
uint32_t moonlab_cuda_state_n_qubits(const moonlab_cuda_state_t* s) {
  uint32_t n = 0;
  return mlb_state_num_qubits(s, &n) == MLB_OK ? n : 0;
}
uint64_t moonlab_cuda_state_dim(const moonlab_cuda_state_t* s) {
  uint64_t d = 0;
  return mlb_state_dim(s, &d) == MLB_OK ? d : 0;
}
moonlab_cuda_status_t moonlab_cuda_apply_1q(moonlab_cuda_state_t* s, uint32_t t, const double m[8]) {
  return mlb_apply_1q(s, t, m);
}
moonlab_cuda_status_t moonlab_cuda_apply_cnot(moonlab_cuda_state_t* s, uint32_t c, uint32_t t) {
  if (c >= 64) return MLB_ERR_INVALID_QUBIT;
  return mlb_apply_mcx(s, 1ull << c, t);
}
moonlab_cuda_status_t moonlab_cuda_apply_2q(moonlab_cuda_state_t* s, uint32_t q0, uint32_t q1, const double m[32]) {
  return mlb_apply_2q(s, q0, q1, m);
}
moonlab_cuda_status_t moonlab_cuda_prob_z(const moonlab_cuda_state_t* s, uint32_t t, double* out) {
  return mlb_prob_one(const_cast<mlb_state*>(s), t, out);
}
moonlab_cuda_status_t moonlab_cuda_norm(const moonlab_cuda_state_t* s, double* out) {
  return mlb_norm_sq(const_cast<mlb_state*>(s), out);
}
moonlab_cuda_status_t moonlab_cuda_apply_x(moonlab_cuda_state_t* s, uint32_t t) {
  return mlb_apply_mcx(s, 0, t);
}
// H as the 2x2 (1/sqrt2)[[1,1],[1,-1]] with the reference's QC_SQRT2_INV.
moonlab_cuda_status_t moonlab_cuda_apply_h(moonlab_cuda_state_t* s, uint32_t t) {
  const double r = 0.70710678118654752440;
  const double h[8] = {r, 0, r, 0, r, 0, -r, 0};
  return mlb_apply_1q(s, t, h);
}
moonlab_cuda_status_t moonlab_cuda_state_copy_to_host(const moonlab_cuda_state_t* s, double* out) {
  return mlb_state_copy_to_host(const_cast<mlb_state*>(s), out);
}
moonlab_cuda_status_t moonlab_cuda_state_copy_from_host(moonlab_cuda_state_t* s, const double* in) {
  return mlb_state_copy_from_host(s, in);
}
moonlab_cuda_status_t moonlab_cuda_apply_mcx(moonlab_cuda_state_t* s, uint64_t cmask, uint32_t t) {
  return mlb_apply_mcx(s, cmask, t);
}
moonlab_cuda_status_t moonlab_cuda_apply_mcz(moonlab_cuda_state_t* s, uint64_t all_mask) {
  return mlb_apply_mcz(s, all_mask);
}
moonlab_cuda_status_t moonlab_cuda_apply_fredkin(moonlab_cuda_state_t* s, uint32_t c, uint32_t t1, uint32_t t2) {
  if (c >= 64) return MLB_ERR_INVALID_QUBIT;
  return mlb_apply_swap(s, 1ull << c, t1, t2);
}
moonlab_cuda_status_t moonlab_cuda_synchronize(moonlab_cuda_state_t* s) { return mlb_synchronize(s); }

int moonlab_cuda_runtime_probe_discrete(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return -2;
  }
  if (n <= 0) return 0;
  int integrated = 0;
  if (cudaDeviceGetAttribute(&integrated, cudaDevAttrIntegrated, 0) != cudaSuccess) return -2;
  return integrated ? -1 : 1;
}

int moonlab_cuda_select_device_for_rank(int local_rank, int* device_id, int* device_count) {
  if (local_rank < 0 || !device_id || !device_count) return MLB_ERR_NO_DEVICE;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return MLB_ERR_NO_DEVICE;
  }
  const int sel = local_rank % n;
  if (cudaSetDevice(sel) != cudaSuccess) return MLB_ERR_DRIVER;
  *device_id = sel;
  *device_count = n;
  return MLB_OK;
}

}  // extern "C"
