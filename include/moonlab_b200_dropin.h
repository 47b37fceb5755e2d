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
 *      calloc'ed as in the reference, so untouched pages cost no memory. ---- */
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
 *      failure: noise model enabled (no exact gradient, as the reference's
 *      exact-or-error contract), an ansatz other than the hardware-efficient
 *      one, or a device error.  The batched variant takes params[B][P] and
 *      writes grads[B][P] with the same codes. ---- */
int moonlab_vqe_gradient(void *solver, const double *parameters, double *gradient_out,
                         size_t num_parameters);
int moonlab_b200_vqe_gradient_batch(void *solver, size_t batch, const double *parameters,
                                    double *gradients_out, size_t num_parameters);

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
