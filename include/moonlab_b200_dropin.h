/*
 * moonlab_b200_dropin.h -- the reference-compatible entry points exported by
 * libmoonlab_b200.so.  Each declaration names the reference interface it
 * replaces (tsotchke/moonlab 1.2.0, paths relative to that project).
 *
 * How it plugs in: the reference core (gates.c, state.c) references these
 * symbols weakly (src/utils/moonlab_weak.h; gates.c:43-50; state.c:89-91,
 * :645-670) and its build links exactly one strong definition of each --
 * either src/quantum/state_gpu.cu + src/backends/cuda_statevec.cu (CUDA on)
 * or src/quantum/gpu_route_cpu_unavailable.c (CUDA off).  Linking or
 * preloading libmoonlab_b200.so in place of those translation units routes
 * every gate_* call on a GPU-backed quantum_state_t to the B200 engine.
 *
 * Types below mirror the reference's public layouts; they are declared here
 * (not included) so this header stands alone.  When compiled together with
 * the reference headers, define MOONLAB_B200_USE_REFERENCE_TYPES and include
 * src/quantum/state.h first.
 */
#ifndef MOONLAB_B200_DROPIN_H
#define MOONLAB_B200_DROPIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Everything declared here is exported from libmoonlab_b200.so (the library is
 * built with -fvisibility=hidden). */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifndef MOONLAB_B200_USE_REFERENCE_TYPES
/* quantum_state_t, src/quantum/state.h:102-131 (field order and types
 * identical; amplitudes is double _Complex* in C). */
typedef struct {
    size_t    num_qubits;
    size_t    state_dim;
    void     *amplitudes;
    uint64_t *measurement_outcomes;
    size_t    num_measurements;
    size_t    max_measurements;
    int       owns_memory;
    void     *gpu_state;
    int       gpu_backend;
} quantum_state_t;
typedef int qs_error_t;  /* QS_* codes, src/quantum/state.h:78-88 */
#endif

typedef struct mlb_state moonlab_cuda_state_t;  /* opaque, cuda_statevec.h:37 */
typedef int moonlab_cuda_status_t;               /* cuda_statevec.h:39-46   */

/* ---- GPU-backed quantum_state_t (src/quantum/state.h:437-464;
 *      reference definitions src/quantum/state_gpu.cu:31-98).
 *      create_gpu accepts 1..33 qubits (reference: 1..31); the host mirror is
 *      calloc'ed as in the reference (the core's gate_* functions refuse a
 *      NULL amplitudes pointer before routing, gates.c:124), and pages of a
 *      block that large are mapped on demand, so the mirror takes host
 *      memory only where sync_to_host has written it. ---- */
qs_error_t quantum_state_create_gpu(size_t num_qubits, quantum_state_t **out_state);
qs_error_t quantum_state_sync_to_host(quantum_state_t *state);
qs_error_t quantum_state_sync_from_host(quantum_state_t *state);

/* ---- gate routing (weak imports in src/quantum/gates.c:43-50; reference
 *      definitions src/quantum/state_gpu.cu:108-199).  0 = ran on GPU,
 *      -1 = not GPU-backed or failed. ---- */
int qsim_gpu_route_hadamard(quantum_state_t *state, int qubit);
int qsim_gpu_route_pauli_x(quantum_state_t *state, int qubit);
int qsim_gpu_route_cnot(quantum_state_t *state, int control, int target);
int qsim_gpu_route_apply_1q_matrix(quantum_state_t *state, int qubit, const double m[8]);
int qsim_gpu_route_apply_2q_matrix(quantum_state_t *state, int q0, int q1, const double m[32]);
int qsim_gpu_route_mcx(quantum_state_t *state, uint64_t control_mask, int target);
int qsim_gpu_route_mcz(quantum_state_t *state, uint64_t all_mask);
int qsim_gpu_route_fredkin(quantum_state_t *state, int control, int t1, int t2);

/* ---- moonlab_cuda_* backend ABI (src/backends/cuda_statevec.h:61-222,
 *      definitions src/backends/cuda_statevec.cu:398-818). ---- */
moonlab_cuda_status_t moonlab_cuda_state_create(uint32_t n_qubits, moonlab_cuda_state_t **out_state);
void     moonlab_cuda_state_free(moonlab_cuda_state_t *state);
uint32_t moonlab_cuda_state_n_qubits(const moonlab_cuda_state_t *state);
uint64_t moonlab_cuda_state_dim(const moonlab_cuda_state_t *state);
moonlab_cuda_status_t moonlab_cuda_apply_1q(moonlab_cuda_state_t *state, uint32_t target, const double m[8]);
moonlab_cuda_status_t moonlab_cuda_apply_cnot(moonlab_cuda_state_t *state, uint32_t control, uint32_t target);
moonlab_cuda_status_t moonlab_cuda_apply_2q(moonlab_cuda_state_t *state, uint32_t q0, uint32_t q1, const double m[32]);
moonlab_cuda_status_t moonlab_cuda_prob_z(const moonlab_cuda_state_t *state, uint32_t target, double *out_prob);
moonlab_cuda_status_t moonlab_cuda_norm(const moonlab_cuda_state_t *state, double *out_norm);
moonlab_cuda_status_t moonlab_cuda_apply_x(moonlab_cuda_state_t *state, uint32_t target);
moonlab_cuda_status_t moonlab_cuda_apply_h(moonlab_cuda_state_t *state, uint32_t target);
moonlab_cuda_status_t moonlab_cuda_state_copy_to_host(const moonlab_cuda_state_t *state, double *out);
moonlab_cuda_status_t moonlab_cuda_state_copy_from_host(moonlab_cuda_state_t *state, const double *in);
moonlab_cuda_status_t moonlab_cuda_apply_mcx(moonlab_cuda_state_t *state, uint64_t control_mask, uint32_t target);
moonlab_cuda_status_t moonlab_cuda_apply_mcz(moonlab_cuda_state_t *state, uint64_t all_mask);
moonlab_cuda_status_t moonlab_cuda_apply_fredkin(moonlab_cuda_state_t *state, uint32_t control, uint32_t t1, uint32_t t2);
moonlab_cuda_status_t moonlab_cuda_synchronize(moonlab_cuda_state_t *state);
/* cuda_statevec.cu:398 -- 1 discrete GPU present, 0 none, -1 integrated, -2 error */
int moonlab_cuda_runtime_probe_discrete(void);
/* cuda_statevec.cu:418 -- device = local_rank mod device count */
int moonlab_cuda_select_device_for_rank(int local_rank, int *device_id, int *device_count);

/* ---- VQE gradient (src/applications/moonlab_export.h:1319, definition
 *      src/applications/moonlab_vqe_export.c:27-42).  solver is the
 *      reference's vqe_solver_t (src/algorithms/vqe.h:545-568).  Returns 0 ok,
 *      -1 NULL argument, -2 num_parameters != ansatz->num_parameters, -3
 *      failure.  Hardware-efficient ansatz, no noise: the batched adjoint
 *      engine.  UCCSD or symmetry-preserving ansatz, no noise: the
 *      reference's exact four-term parameter-shift rule (vqe.c:2072-2140),
 *      the shifted energies on the device.  A noise model without the
 *      solver's allow_stochastic_gradient: -3 (exact-or-error, vqe.c:2060-2066).
 *      A CUSTOM ansatz, or a noisy solver that opted into stochastic
 *      parameter shift: the reference's own vqe_compute_gradient, found at
 *      run time in the process (-3 when absent).  The batched variant takes
 *      params[B][P] and writes grads[B][P] with the same codes. ---- */
int moonlab_vqe_gradient(void *solver, const double *parameters, double *gradient_out,
                         size_t num_parameters);
int moonlab_b200_vqe_gradient_batch(void *solver, size_t batch, const double *parameters,
                                    double *gradients_out, size_t num_parameters);

/* ---- Quantum geometry verbs (src/applications/moonlab_vqe_export.c:53-100,
 *      ABI 0.7.0).  Same codes as moonlab_vqe_gradient.  qgt_out / berry_out:
 *      num_parameters^2 doubles, row-major, filled as vqe_compute_qgt and
 *      vqe_compute_berry_curvature fill them (src/algorithms/vqe_qng.c:166-232);
 *      direction_out = (g + regularization I)^-1 gradient by the same
 *      partial-pivot elimination (vqe_qng.c:236-282; a pivot below 1e-300 is
 *      singular: -3, and the caller falls back to the plain gradient as with
 *      the reference).  Hardware-efficient ansatz: psi and the P derivative
 *      states as one device batch and an FP64 Gram kernel (mlb_hea_geometry).
 *      Other ansaetze: the reference's own vqe_compute_qgt /
 *      vqe_compute_berry_curvature / vqe_natural_gradient_direction, found at
 *      run time in the process (-3 when absent). ---- */
int moonlab_vqe_qgt(void *solver, const double *parameters, double *qgt_out, size_t num_parameters);
int moonlab_vqe_berry_curvature(void *solver, const double *parameters, double *berry_out,
                                size_t num_parameters);
int moonlab_vqe_natural_gradient(void *solver, const double *parameters, const double *gradient,
                                 double regularization, double *direction_out, size_t num_parameters);

/* ---- single-qubit gate fusion (src/optimization/fusion/fusion.h:73-458,
 *      definitions src/optimization/fusion/fusion.c:127-394).
 *      Same records, validation (-1 on a bad qubit or a == b) and run-length
 *      rule in fuse_compile (FUSED_1Q products, fusion.c:247-292).
 *      fuse_execute queues the whole list on the engine in one call: on a
 *      GPU-backed state its own device state; on a host state a temporary
 *      device state (uploaded, run, read back).  QS_ERROR_INVALID_STATE on
 *      NULL arguments, QS_ERROR_INVALID_DIMENSION when the state has fewer
 *      qubits than the circuit, as the reference. ---- */
#ifndef MOONLAB_B200_USE_REFERENCE_TYPES
typedef enum {
    FUSE_GATE_H = 0, FUSE_GATE_X, FUSE_GATE_Y, FUSE_GATE_Z, FUSE_GATE_S, FUSE_GATE_SDG,
    FUSE_GATE_T, FUSE_GATE_TDG, FUSE_GATE_PHASE, FUSE_GATE_RX, FUSE_GATE_RY, FUSE_GATE_RZ,
    FUSE_GATE_U3, FUSE_GATE_FUSED_1Q, FUSE_GATE_CNOT, FUSE_GATE_CZ, FUSE_GATE_CY, FUSE_GATE_SWAP,
    FUSE_GATE_CPHASE, FUSE_GATE_CRX, FUSE_GATE_CRY, FUSE_GATE_CRZ
} fuse_gate_kind_t;
typedef struct {            /* fusion.h:99-104; u is complex_t u[2][2] in C */
    int    kind;
    int    q[2];
    double p[3];
    double u[2][2][2];
} fuse_gate_t;
typedef struct fuse_circuit_t fuse_circuit_t;
typedef struct {
    size_t original_gates;
    size_t fused_gates;
    size_t merges_applied;
} fuse_stats_t;
#endif
fuse_circuit_t *fuse_circuit_create(size_t num_qubits);
void   fuse_circuit_free(fuse_circuit_t *c);
size_t fuse_circuit_len(const fuse_circuit_t *c);
size_t fuse_circuit_num_qubits(const fuse_circuit_t *c);
int fuse_append_h(fuse_circuit_t *c, int q);
int fuse_append_x(fuse_circuit_t *c, int q);
int fuse_append_y(fuse_circuit_t *c, int q);
int fuse_append_z(fuse_circuit_t *c, int q);
int fuse_append_s(fuse_circuit_t *c, int q);
int fuse_append_sdg(fuse_circuit_t *c, int q);
int fuse_append_t(fuse_circuit_t *c, int q);
int fuse_append_tdg(fuse_circuit_t *c, int q);
int fuse_append_phase(fuse_circuit_t *c, int q, double theta);
int fuse_append_rx(fuse_circuit_t *c, int q, double theta);
int fuse_append_ry(fuse_circuit_t *c, int q, double theta);
int fuse_append_rz(fuse_circuit_t *c, int q, double theta);
int fuse_append_u3(fuse_circuit_t *c, int q, double theta, double phi, double lambda);
int fuse_append_cnot(fuse_circuit_t *c, int ctrl, int tgt);
int fuse_append_cz(fuse_circuit_t *c, int ctrl, int tgt);
int fuse_append_cy(fuse_circuit_t *c, int ctrl, int tgt);
int fuse_append_swap(fuse_circuit_t *c, int a, int b);
int fuse_append_cphase(fuse_circuit_t *c, int ctrl, int tgt, double theta);
int fuse_append_crx(fuse_circuit_t *c, int ctrl, int tgt, double theta);
int fuse_append_cry(fuse_circuit_t *c, int ctrl, int tgt, double theta);
int fuse_append_crz(fuse_circuit_t *c, int ctrl, int tgt, double theta);
fuse_circuit_t *fuse_compile(const fuse_circuit_t *src, fuse_stats_t *stats);
qs_error_t fuse_execute(const fuse_circuit_t *c, quantum_state_t *state);
/* The engine ops fuse_execute queues for a fusion circuit on num_qubits
 * qubits: ops is an mlb_op_t array of `capacity` records (moonlab_b200.h), or
 * NULL to count only into *num_ops.  No counterpart in the reference: for
 * callers that keep their own engine states (mlb_apply_ops). */
int mlb_fuse_circuit_ops(const fuse_circuit_t *c, uint32_t num_qubits, void *ops, size_t capacity,
                         size_t *num_ops);

/* ---- scheduler backend plug-in (src/distributed/scheduler.h:225-262,
 *      registry scheduler.c:283-305).
 * moonlab_b200_backend_execute is a moonlab_backend_execute_fn: it reads the
 * job through the reference's moonlab_job_to_json, runs it on the B200 with
 * the "simulator" backend's semantics (mlb_job_run) and fills the
 * moonlab_job_results_t the scheduler passes in (outcomes and
 * worker_seconds malloc'ed, freed by the scheduler).  Returns
 * MOONLAB_SCHED_OK (0), MOONLAB_SCHED_BAD_ARG (-501), MOONLAB_SCHED_OOM
 * (-502) or MOONLAB_SCHED_INTERNAL (-503).  ctx: NULL (device 0) or a
 * pointer to an int device ordinal.
 * moonlab_b200_register_backend registers it under the name "b200" with the
 * scheduler loaded in the process (found with dlsym, so this library does
 * not link against the reference); after it, moonlab_job_set_backend(job,
 * "b200") routes moonlab_scheduler_run to the GPU.  Returns the registry's
 * code, or MOONLAB_SCHED_BACKEND_NOT_FOUND (-506) when no scheduler is
 * loaded.  A host that opened the reference library privately (RTLD_LOCAL,
 * as ctypes does by default) passes its moonlab_register_backend and
 * moonlab_job_to_json to moonlab_b200_register_backend_with instead.
 * moonlab_b200_release_backend_state frees the cached device state. */
int moonlab_b200_backend_execute(const void *job, void *results, void *ctx);
int moonlab_b200_register_backend(void);
int moonlab_b200_register_backend_with(void *register_fn, void *job_to_json_fn);
void moonlab_b200_release_backend_state(void);

/* The engine handle behind a GPU-backed quantum_state_t (for callers that
 * want the engine's FP64 reductions, sampling and collapse directly). */
struct mlb_state *moonlab_b200_engine_of(quantum_state_t *state);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* MOONLAB_B200_DROPIN_H */
