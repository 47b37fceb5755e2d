/*
 * moonlab_b200.h -- C ABI of the B200 (sm_100a) dense state-vector engine.
 *
 * Plain C types only: pointers, sizes, integers, doubles.  Every entry point
 * returns an mlb_status_t (0 = success, negative = error) unless stated.
 * This is the engine's own surface; the reference-compatible drop-in symbols
 * (quantum_state_create_gpu, qsim_gpu_route_*, moonlab_cuda_*,
 * moonlab_vqe_gradient, the "b200" scheduler backend) are declared in
 * moonlab_b200_dropin.h and are implemented on top of this one.
 *
 * State layout in HBM: 2^n amplitudes, interleaved (re, im), qubit 0 = the
 * least-significant index bit -- the quantum_state_t.amplitudes layout of the
 * reference (src/quantum/state.h:102-131).  complex128 states hold doubles,
 * complex64 states floats.
 *
 * Threading: a state is not thread-safe (as quantum_state_t,
 * src/quantum/state.h:98-100); distinct states may be used from distinct
 * threads.  Gate calls are asynchronous: they are queued on the host and run
 * on the state's stream in fused tile passes at the next read, flush or
 * synchronize.
 */
#ifndef MOONLAB_B200_H
#define MOONLAB_B200_H

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

/* Status codes.  0 .. -5 carry the meaning of moonlab_cuda_status_t
 * (src/backends/cuda_statevec.h:39-46) so the drop-in layer passes them
 * through unchanged. */
typedef enum {
    MLB_OK                = 0,
    MLB_ERR_OUT_OF_MEMORY = -1,
    MLB_ERR_NO_DEVICE     = -2,
    MLB_ERR_DRIVER        = -3,
    MLB_ERR_INVALID_QUBIT = -4,
    MLB_ERR_NUM_QUBITS    = -5,
    MLB_ERR_INVALID_ARG   = -6,
    MLB_ERR_TIMEOUT       = -7,  /* a bounded device-side wait gave up */
    MLB_ERR_BUSY          = -8,  /* admission refused (HBM budget / slots) */
    MLB_ERR_NOT_SUPPORTED = -9
} mlb_status_t;

typedef enum { MLB_C128 = 0, MLB_C64 = 1 } mlb_dtype_t;

/* Execution modes for queued gates.  A new state starts in MLB_EXEC_TILED
 * (complex128) or MLB_EXEC_FUSED (complex64). */
typedef enum {
    MLB_EXEC_TILED = 0,  /* gates grouped into shared-memory tile passes */
    MLB_EXEC_EAGER = 1,  /* one full-state kernel per gate (the per-gate path) */
    MLB_EXEC_FUSED = 2   /* complex64 states: gates fused into dense k<=5-qubit blocks on the
                            tensor cores; states under 13 qubits and ops on more than 5 qubits
                            run as tile passes */
} mlb_exec_mode_t;

/* Gate operation kinds understood by the engine (mlb_op_t.kind). */
typedef enum {
    MLB_OP_1Q      = 0, /* 2x2 matrix m[0..7] on target, if (idx & cmask) == cmask   */
    MLB_OP_2Q      = 1, /* 4x4 matrix m[0..31] on (target = low bit, target2), cmask */
    MLB_OP_DIAG1   = 2, /* diag(m[0]+i m[1], m[2]+i m[3]) on target, cmask           */
    MLB_OP_X       = 3, /* swap the target pair where (idx & cmask) == cmask        */
    MLB_OP_SWAP    = 4, /* swap bits target <-> target2 where cmask holds           */
    MLB_OP_ZZ      = 5, /* amp *= (m[0],m[1]) if bit(target)==bit(target2) else (m[2],m[3]) */
    MLB_OP_PHASE   = 6, /* amp *= (m[0],m[1]) where (idx & cmask) == cmask          */
    MLB_OP_DENSE   = 7  /* dense 2^k x 2^k block (fused path); internal               */
} mlb_op_kind_t;

typedef struct {
    int32_t  kind;
    int32_t  target;
    int32_t  target2;
    int32_t  reserved;
    uint64_t cmask;
    double   m[32];
} mlb_op_t;

typedef struct mlb_state mlb_state_t;

/* ---- device / lifecycle ---------------------------------------------- */
int  mlb_device_count(int *count);
/* The device's FP64 tensor-core throughput in TFLOP/s, measured now: a
 * register-only probe of mma.sync m8n8k4 f64 (the instruction of the dense
 * complex128 segments), 16 warps per SM, best of three launches.  For
 * rooflines; no counterpart in the reference. */
int  mlb_fp64_tensor_peak(int device, double *tflops);
int  mlb_state_create(uint32_t num_qubits, int dtype, int device, mlb_state_t **out);
void mlb_state_free(mlb_state_t *s);
int  mlb_state_num_qubits(const mlb_state_t *s, uint32_t *out);
int  mlb_state_dim(const mlb_state_t *s, uint64_t *out);
int  mlb_state_dtype(const mlb_state_t *s, int *out);
/* The state's device buffer (flushes first).  After a reset, tile passes run
 * only over the tiles that can hold nonzero amplitudes; once this pointer has
 * been handed out, writes through it cannot be followed, so every later pass
 * of this state runs over every tile. */
int  mlb_state_device_ptr(mlb_state_t *s, void **out);
int  mlb_state_set_stream(mlb_state_t *s, void *cuda_stream); /* NULL = own stream */
int  mlb_state_stream(const mlb_state_t *s, void **cuda_stream); /* the stream kernels run on */
int  mlb_state_set_exec_mode(mlb_state_t *s, int mode);
int  mlb_state_reset(mlb_state_t *s);                     /* |0...0> */
int  mlb_state_copy_to_host(mlb_state_t *s, void *host);  /* 2^n (re,im) of the dtype */
int  mlb_state_copy_from_host(mlb_state_t *s, const void *host);
int  mlb_state_copy(mlb_state_t *dst, mlb_state_t *src); /* same n; dtype may differ */
int  mlb_flush(mlb_state_t *s);
int  mlb_synchronize(mlb_state_t *s);

/* ---- gates (queued) ---------------------------------------------------- */
int  mlb_apply_op(mlb_state_t *s, const mlb_op_t *op);
int  mlb_apply_ops(mlb_state_t *s, const mlb_op_t *ops, size_t num_ops);
int  mlb_apply_1q(mlb_state_t *s, uint32_t target, const double m[8]);
int  mlb_apply_2q(mlb_state_t *s, uint32_t q0, uint32_t q1, const double m[32]);
int  mlb_apply_controlled_1q(mlb_state_t *s, uint64_t control_mask, uint32_t target,
                             const double m[8]);
int  mlb_apply_mcx(mlb_state_t *s, uint64_t control_mask, uint32_t target);
int  mlb_apply_mcz(mlb_state_t *s, uint64_t all_mask);
int  mlb_apply_swap(mlb_state_t *s, uint64_t control_mask, uint32_t q0, uint32_t q1);
int  mlb_apply_zz(mlb_state_t *s, uint32_t q0, uint32_t q1, double theta);

/* ---- FP64 reductions (one HBM pass each) ------------------------------- */
int  mlb_norm_sq(mlb_state_t *s, double *out);
int  mlb_prob_one(mlb_state_t *s, uint32_t qubit, double *out);
int  mlb_prob_one_all(mlb_state_t *s, double *out_n);          /* P1 of every qubit */
int  mlb_expect_z_all(mlb_state_t *s, double *out_n);          /* 1 - 2 P1 */
/* P(qubit = 1) bit-identical to measurement_probability_one (measurement.c:73):
 * the reference's left-to-right fused sum, reproduced exactly (two passes). */
int  mlb_prob_one_exact(mlb_state_t *s, uint32_t qubit, double *out);
int  mlb_correlation_zz(mlb_state_t *s, uint32_t q1, uint32_t q2, double *out);
int  mlb_expect_pauli(mlb_state_t *s, uint64_t xmask, uint64_t zmask, double *out);
int  mlb_expect_pauli_sum(mlb_state_t *s, size_t num_terms, const uint64_t *xmasks,
                          const uint64_t *zmasks, const double *coeffs, double *out);
/* mlb_prob_one_all_noalloc: the one-pass reduction of mlb_prob_one_all and
 * mlb_norm_sq, run on amplitudes the caller owns and written to device
 * memory the caller owns.  It allocates nothing.  No counterpart in the
 * reference (its reductions read host memory).
 *   amp_device  2^num_qubits amplitudes of `dtype` (MLB_C128 / MLB_C64) in
 *               memory of the current device;
 *   out_device  num_qubits + 1 doubles on the same device: P(qubit q = 1)
 *               for q < num_qubits, then the squared norm;
 *   stream      a cudaStream_t of the current device (NULL: default stream).
 *               The call only enqueues two kernels; out_device is ready when
 *               the stream has run them.
 * Meant for callers that may not allocate device memory: a process that has
 * reserved all of HBM up front under a fixed budget (a serving process, or a
 * host framework whose own allocator owns the device), and latency-critical
 * loops where cudaMalloc / cudaFree would stall on device synchronisation.
 * Its scratch is one fixed array per device inside this library, 1,163,264
 * bytes, which sets the limit: num_qubits 1..30, else MLB_ERR_NUM_QUBITS.
 * All calls on a device share that array: two calls whose kernels overlap on
 * the GPU (different streams, or different host threads) race and return
 * wrong values, so order them on one stream or synchronise between them.
 * Each call writes every scratch entry it reads; nothing needs clearing.
 * The first call on a device does a one-time set-up (it looks up the
 * array's address and the SM count); make that first call before any stream
 * capture on that device.  The looked-up address belongs to the device's
 * current context: the set-up does not survive cudaDeviceReset (or any
 * other teardown of the primary context), after which this entry point must
 * not be called again in the process.  Errors: MLB_ERR_INVALID_ARG for null,
 * misaligned or non-device buffers and a bad dtype. */
int  mlb_prob_one_all_noalloc(const void *amp_device, int dtype, uint32_t num_qubits,
                              double *out_device, void *stream);
/* probability vector; rule 0 = cabs(a)^2 (measurement.c:140),
 * rule 1 = re*re + im*im (moonlab_qgtl_backend.c:199-210).
 * out_host may be NULL when out_device is given (device pointer, 2^n doubles). */
int  mlb_probabilities(mlb_state_t *s, int rule, double *out_host, void *out_device);

/* ---- sampling and collapse (bit-exact vs the reference given uniforms) -- */
enum { MLB_SAMPLE_CDF_GE = 0,   /* measurement_sample: first i with cdf_i >= u      */
       MLB_SAMPLE_CUM_GT = 1 }; /* measurement_all_qubits: first i with u < cum_i  */
int  mlb_sample(mlb_state_t *s, int rule, const double *uniforms, size_t num,
                uint64_t *outcomes);
/* measurement_single_qubit semantics; *outcome = -1 when the kept norm is tiny */
int  mlb_measure_qubit(mlb_state_t *s, uint32_t qubit, double u, int *outcome);
/* quantum_measure (computational basis) semantics */
int  mlb_quantum_measure(mlb_state_t *s, uint32_t qubit, double u, int *outcome,
                         double *probability);
/* measurement_all_qubits: sample (rule CUM_GT) and collapse to the basis state */
int  mlb_measure_all(mlb_state_t *s, double u, uint64_t *outcome);
int  mlb_normalize(mlb_state_t *s, double *norm_out);

/* ---- circuits ------------------------------------------------------------ */
/* Circuit gate record.  type: the QGTL gate enum 0..13
 * (moonlab_qgtl_backend.h:57-72; CY composed as S.CNOT.Sdg like
 * moonlab_qgtl_backend.c:138-144) plus Sdg = 20, Tdg = 21, Phase = 22,
 * CPhase = 23, CRX = 24, CRY = 25, CRZ = 26 (gates.c:345-887) and
 * ZZ(theta) = 27 (exp(-i theta/2 Z Z), qaoa.c:745-753).  Two-qubit records
 * use `control` as the control (or first qubit) and `target` as the target. */
typedef struct {
    int32_t type;
    int32_t target;
    int32_t control;   /* control (CNOT/CY/CZ), qubit1 (SWAP), second qubit (ZZ) */
    int32_t reserved;
    double  theta;
} mlb_gate_t;
enum { MLB_GATE_SDG = 20, MLB_GATE_TDG = 21, MLB_GATE_PHASE = 22, MLB_GATE_CPHASE = 23,
       MLB_GATE_CRX = 24, MLB_GATE_CRY = 25, MLB_GATE_CRZ = 26, MLB_GATE_ZZ = 27 };

/* Translate gate records into engine ops exactly as the reference's gate_*
 * functions build their GPU-route matrices (host libm cos/sin/cexp). */
int  mlb_gates_to_ops(const mlb_gate_t *gates, size_t num_gates, uint32_t num_qubits,
                      mlb_op_t *ops_out, size_t *num_ops_out);
int  mlb_run_gates(mlb_state_t *s, const mlb_gate_t *gates, size_t num_gates);

/* ---- scheduler jobs -------------------------------------------------------
 * A job as the reference's scheduler holds it (src/distributed/scheduler.c:
 * num_qubits, gate records of the QGTL enum, total shots, worker fan-out,
 * base seed).  mlb_job_parse_json reads the text of moonlab_job_to_json
 * (scheduler.c:492-537; theta printed with %.17g, so it round-trips
 * exactly).  Pass gates = NULL to learn the gate count; with a buffer that
 * is too small the call returns MLB_ERR_INVALID_ARG and sets *num_gates to
 * the count needed.  Malformed text: MLB_ERR_INVALID_ARG. */
typedef struct {
    int32_t  num_qubits;
    int32_t  num_shots;
    int32_t  num_workers;
    int32_t  reserved;
    uint64_t rng_seed;
} mlb_job_desc_t;
int  mlb_job_parse_json(const char *json, mlb_job_desc_t *desc, mlb_gate_t *gates,
                        size_t capacity, size_t *num_gates);
/* Circuit text: the "moonlab-circuit v1" line format of
 * moonlab_qgtl_circuit_serialize / moonlab_qgtl_circuit_deserialize
 * (moonlab_qgtl_backend.h:190-205, moonlab_qgtl_backend.c:319-506).
 * mlb_circuit_parse_text reads it into gate records (types 0..13; for
 * CNOT/CY/CZ/SWAP the line is "<NAME> <target> <control>") with the
 * deserializer's rules: len = 0 reads a NUL-terminated string, and with
 * len > 0 a NUL inside the extent is invalid; "NUM_QUBITS n" (1..32) must
 * be the first line that is not blank or a '#' comment; a line over 255
 * bytes, an unknown name, a missing field, a qubit out of range or a
 * control equal to its target is invalid (MLB_ERR_INVALID_ARG).  Records
 * of one-qubit gates get control = -1.  Pass gates = NULL to learn the
 * count; with a buffer that is too small the call returns
 * MLB_ERR_INVALID_ARG and sets *num_gates to the count needed.
 * mlb_circuit_format_text writes the serializer's text byte for byte
 * (theta with %.17g, so it round-trips exactly); a record type without a
 * name in the format (20..27) gives MLB_ERR_NOT_SUPPORTED.  buf = NULL,
 * capacity = 0 asks for the length; too small a buffer gives
 * MLB_ERR_INVALID_ARG with *written = the capacity needed (text + NUL).
 * Replaces moonlab_qgtl_circuit_deserialize / _serialize (moonlab_qgtl_backend.h:
 * 227-252) for callers that go straight to mlb_run_gates or mlb_job_run. */
int  mlb_circuit_parse_text(const char *text, size_t len, uint32_t *num_qubits, mlb_gate_t *gates,
                            size_t capacity, size_t *num_gates);
int  mlb_circuit_format_text(uint32_t num_qubits, const mlb_gate_t *gates, size_t num_gates, char *buf,
                             size_t capacity, size_t *written);
/* Run a job with the semantics of the scheduler's default "simulator"
 * backend (simulator_backend_execute, scheduler.c:194-239): workers =
 * min(num_workers, num_shots), worker w takes shots [w S / W, (w+1) S / W)
 * and draws its uniforms from xorshift64 seeded with
 * splitmix64(rng_seed ^ (w << 32)) (moonlab_qgtl_backend.c:158-167,
 * :226-240); each shot is measurement_all_qubits on the circuit's output
 * state.  Here the circuit runs once, on `device`, in complex128, and all
 * shots are sampled from that state; outcomes[num_shots] are bit-identical
 * to the reference's for a non-zero rng_seed (a zero seed takes the clock,
 * as the reference does).  *workers_used and *seconds (wall time of the
 * whole job) may be NULL. */
int  mlb_job_run(const mlb_job_desc_t *desc, const mlb_gate_t *gates, size_t num_gates,
                 int device, uint64_t *outcomes, int *workers_used, double *seconds);

/* ---- serving: a continuous-batching request loop on one GPU --------------
 * mlb_server_submit queues a request and returns at once with a ticket.
 * num_workers threads admit queued requests in arrival order whenever a
 * worker and HBM budget are free (first fit; a request waiting longer than
 * 0.5 s holds back later ones), so requests that arrive while others run
 * start without waiting for a batch to finish and overlap on the device.
 * Device states are pooled per (qubits, dtype) and count against the
 * budget (0 = 80 % of the device's free memory at creation).  A request's
 * shots follow moonlab_qgtl_execute (moonlab_qgtl_backend.c:218-240):
 * uniforms from xorshift64(rng_seed), each shot measurement_all_qubits(u) on
 * the circuit's output state (rng_seed 0 takes the clock).  Results do not
 * depend on the other requests in flight.  Times in mlb_request_info_t are
 * seconds since the server was created.  Small requests (<= 12 qubits
 * complex128, <= 13 complex64) skip the state pool: the waiting ones of a
 * dtype run together in one launch, one thread block per circuit with its
 * state in shared memory.  mlb_server_wait blocks up to
 * timeout_ms (< 0: no limit; MLB_ERR_TIMEOUT when it runs out), copies the
 * outcomes (capacity >= num_shots), releases the ticket and returns the
 * request's status.  mlb_server_destroy cancels requests not yet admitted
 * (MLB_ERR_BUSY), lets running ones finish and frees everything; no thread
 * may be inside mlb_server_wait when it is called. */
typedef struct mlb_server mlb_server_t;
typedef struct {
    uint32_t          num_qubits;
    int32_t           dtype;        /* MLB_C128 or MLB_C64 */
    const mlb_gate_t *gates;        /* copied at submit */
    size_t            num_gates;
    uint32_t          num_shots;
    uint32_t          reserved;
    uint64_t          rng_seed;
} mlb_request_t;
typedef struct {
    int32_t  status;
    uint32_t num_qubits;
    int32_t  dtype;
    uint32_t num_shots;
    double   submit_s, admit_s, done_s;
} mlb_request_info_t;
typedef struct {
    uint64_t submitted, completed, failed, pending, running, peak_running;
    uint64_t reserved_bytes, peak_reserved_bytes, budget_bytes;
    uint64_t small_batches, small_requests;  /* size-class launches and the requests they ran */
    uint64_t plan_cache_hits;                /* requests whose plan came from a state's cache */
} mlb_server_stats_t;
int  mlb_server_create(int device, size_t hbm_budget_bytes, int num_workers, mlb_server_t **out);
int  mlb_server_submit(mlb_server_t *s, const mlb_request_t *req, uint64_t *ticket);
int  mlb_server_wait(mlb_server_t *s, uint64_t ticket, int timeout_ms, uint64_t *outcomes,
                     size_t capacity, mlb_request_info_t *info);
int  mlb_server_get_stats(mlb_server_t *s, mlb_server_stats_t *out);
void mlb_server_destroy(mlb_server_t *s);

/* ---- persistent request loop for small circuits (a mailbox) ---------------
 * One long-running launch serves small requests (<= 12 qubits complex128,
 * <= 13 complex64, one dtype per mailbox) as they are posted: submit copies
 * the request into a device-memory ring slot and publishes it; `ctas`
 * thread blocks (one SM each; default 8, the rest of the GPU stays free for
 * other work) claim published requests, run them with the state in shared
 * memory and write the outcomes into mapped host memory, which
 * mlb_mailbox_wait polls.  Shots follow moonlab_qgtl_execute exactly as in
 * mlb_server_*: bit-identical outcomes for a non-zero rng_seed.  The loop's
 * waits are bounded: after idle_ms (default 1000) without a request its
 * blocks exit and the launch ends with MLB_ERR_TIMEOUT (counted in
 * idle_exits); the next submit, or a waiter whose request is pending,
 * relaunches it.  submit returns MLB_ERR_BUSY when all `slots` (default 64)
 * hold unwaited tickets; a request with more than max_ops ops after fusion
 * (default 2048) or max_shots shots (default 4096) is refused
 * (MLB_ERR_INVALID_ARG).  wait: timeout_ms < 0 waits without limit, else
 * MLB_ERR_TIMEOUT when it runs out (the ticket stays valid).  free stops the
 * loop (it finishes the request in hand) and releases everything; tickets
 * not yet waited are dropped. */
typedef struct mlb_mailbox mlb_mailbox_t;
typedef struct {
    int32_t  dtype;      /* MLB_C128 or MLB_C64 */
    int32_t  device;
    int32_t  ctas;       /* 0: 8 */
    uint32_t slots;      /* 0: 64 */
    uint32_t max_ops;    /* 0: 2048 */
    uint32_t max_shots;  /* 0: 4096 */
    double   idle_ms;    /* 0: 1000 */
} mlb_mailbox_config_t;
typedef struct {
    uint64_t submitted, completed;
    uint64_t launches;    /* launches of the request loop */
    uint64_t idle_exits;  /* launches that ended on the idle limit (MLB_ERR_TIMEOUT) */
    uint64_t running;     /* 1 while a launch is live */
} mlb_mailbox_stats_t;
int mlb_mailbox_create(const mlb_mailbox_config_t *cfg, mlb_mailbox_t **out);
int mlb_mailbox_submit(mlb_mailbox_t *mb, const mlb_request_t *req, uint64_t *ticket);
int mlb_mailbox_wait(mlb_mailbox_t *mb, uint64_t ticket, int timeout_ms, uint64_t *outcomes, size_t capacity);
int mlb_mailbox_get_stats(mlb_mailbox_t *mb, mlb_mailbox_stats_t *out);
int mlb_mailbox_free(mlb_mailbox_t *mb);

/* ---- control-plane front end ----------------------------------------------
 * The request execution of the reference's control server
 * (src/control/control_plane.c:598-770) on the device loop: one request
 * frame in (the bytes after the AUTH line, if any; the transport, TLS,
 * AUTH/HMAC, rate limits, METRICS and admission hooks stay the server's),
 * its response frame out (control_plane.h:8-33):
 *   "HEALTH\n"                        -> "OK alive\n"
 *   "CIRCUIT <N>\n" + N bytes of text -> "OK <2^n>\n" + 2^n little-endian
 *       doubles, re*re + im*im of the output state (moonlab_qgtl_backend.c:199-210)
 *   "SHOTS <k> <N>\n" + N bytes       -> "SAMPLES <k>\n" + k little-endian
 *       uint64 outcomes drawn as moonlab_qgtl_execute draws them
 *   failure                           -> "ERR <code> <message>\n" with the
 *       reference's codes and messages (-401 out of range, -404 malformed
 *       frame, -405 rejected: "deserialize" / "execute").
 * The text is "moonlab-circuit v1" (mlb_circuit_parse_text); limits as the
 * reference's: body 1..4 MiB, shots 1..2^20, and a qubit cap
 * (MOONLAB_CONTROL_MAX_QUBITS there): max_qubits, 0 = 30 (the reference's
 * ceiling; its default is 24), at most 33.  SHOTS requests run in a
 * continuous-batching server (mlb_server_*, created at the first SHOTS
 * request with hbm_budget_bytes and num_workers) in complex128, so many
 * overlap on the device; CIRCUIT requests run one at a time on a complex128
 * state of their own, outside the server's budget.  Shots take their seed
 * from the clock, as the reference's server does, unless
 * mlb_control_set_seed gave a fixed non-zero one (then outcomes equal
 * moonlab_qgtl_execute's with that seed).  mlb_control_handle is
 * thread-safe; it returns MLB_OK whenever it produced a response frame (ERR
 * frames included) in *response (free with mlb_control_free).  No
 * counterpart in the reference's C API: it is the body of its connection
 * handler. */
typedef struct mlb_control mlb_control_t;
int  mlb_control_create(int device, size_t hbm_budget_bytes, int num_workers, uint32_t max_qubits,
                        mlb_control_t **out);
int  mlb_control_set_seed(mlb_control_t *c, uint64_t seed);
int  mlb_control_handle(mlb_control_t *c, const void *request, size_t request_len, void **response,
                        size_t *response_len);
void mlb_control_free(void *response);
void mlb_control_destroy(mlb_control_t *c);

/* Plan statistics of the last flush: passes launched and ops applied. */
typedef struct {
    uint64_t passes;
    uint64_t ops;
    uint64_t dense_blocks;   /* fused complex64 blocks, or complex128 segments run as dense
                                matrices on the FP64 tensor cores */
    uint64_t bytes_moved;    /* HBM bytes of the tiles the launched passes ran over (2 x state
                                bytes per pass, less the tiles skipped as all-zero) */
    uint64_t kernel_launches;
    uint64_t segments;       /* shared-memory register-group round trips over all passes */
    double   gpu_ms;         /* device time of the flush's kernels (timing enabled), else 0 */
    uint64_t plan_cache_hit; /* 1 when the plan came from the state's plan cache */
    uint64_t dense_amps;     /* complex128: amplitudes times dense segments applied to them
                                (FP64 tensor-core work = 96 flops each) */
} mlb_flush_stats_t;
int  mlb_last_flush_stats(mlb_state_t *s, mlb_flush_stats_t *out);
/* Plan cache for repeated circuit shapes (tiled mode): up to `entries` plans
 * are kept per state, keyed by the shape of the flushed ops (kinds, qubits,
 * controls, real or complex 1-qubit matrices -- not the angles).  A flush
 * whose shape was seen before skips planning: it patches this circuit's
 * matrices into the cached op program and replays the passes' launches as
 * one CUDA graph (captured at the shape's first replay).  Results are
 * identical with and without the cache.  0 entries (default) = off. */
int  mlb_state_set_plan_cache(mlb_state_t *s, size_t entries);
/* complex128 tiled mode: run each register segment that fits (4 register
 * qubits in a 13-qubit tile, at most 4 conditioning qubits outside them) as a
 * dense 16x16 complex matrix on the FP64 tensor cores (mma.sync f64), the
 * others gate by gate.  On (1) by default; 0 runs every segment gate by gate.
 * Queued ops are flushed first.  Results agree to rounding (~1e-15 per
 * amplitude per pass).  No counterpart in the reference, whose CPU path has
 * no such choice. */
int  mlb_state_set_dense(mlb_state_t *s, int on);
/* Record CUDA events around each flush's kernels on the state's stream;
 * mlb_last_flush_stats then reports their elapsed device time (synchronizes). */
int  mlb_state_set_timing(mlb_state_t *s, int enable);
/* Test hook for the fused path's bounded waits (complex64 states in
 * MLB_EXEC_FUSED): the next fused flush runs its first pass with CTA 0's
 * first operand-image copy not requested and every wait limited to 20 ms
 * instead of 2 s.  That CTA's waits run out with no copy and no tensor-core
 * work in flight, it frees its tensor memory and returns, and the flush's
 * synchronize reports MLB_ERR_TIMEOUT; the state's contents are then
 * undefined but the state and the device stay usable (reset and rerun).
 * Queued ops are flushed first.  No counterpart in the reference. */
int  mlb_test_fused_skip_copy(mlb_state_t *s);
/* Plan ops exactly as a flush would, on the host only (no device needed):
 * reports the passes and algorithmic bytes a flush of these ops launches.
 * fuse1q != 0 applies a flush's op fusion first: runs of uncontrolled
 * 1-qubit ops on one qubit are merged (fusion.c:247-292), and a
 * CNOT . diagonal . CNOT sandwich on the same (control, target), the
 * reference's exp(-i g J Z Z) (qaoa.c:598-602), becomes one ZZ op. */
int  mlb_plan_ops(const mlb_op_t *ops, size_t num_ops, uint32_t num_qubits, int dtype,
                  int fuse1q, mlb_flush_stats_t *out);
/* The tile-pass plan a flush of these ops runs (host only), for inspection
 * and host replay: the ops after op fusion (fuse1q as for mlb_plan_ops) in
 * execution order, the passes over them and each pass's register-group
 * segments.  A pass's tile is qubits 0..num_low-1 plus high[0..num_high-1]
 * (tile bit num_low + i <-> qubit high[i]); every op of the pass has its
 * non-diagonal targets in the tile, and a mode-0 segment's ops have theirs
 * among its register bits (tile bits bits[0..nbits-1]).  mode: 0 gate by
 * gate, 1 one generic 4x4 op in shared memory, 2 a dense 16x16 complex128
 * matrix on the FP64 tensor cores (dtype MLB_C128 with dense segments on,
 * as a state flushes by default).  Segments index the ops [op_begin,
 * op_end) of the execution order.  Call with NULL buffers to learn the
 * sizes; a buffer too small gives MLB_ERR_INVALID_ARG. */
typedef struct {
    uint8_t  high[16];
    uint8_t  num_low;
    uint8_t  num_high;
    uint8_t  reserved[2];
    uint32_t seg_begin;
    uint32_t num_segments;
} mlb_tile_pass_t;
typedef struct {
    int32_t  mode;
    int32_t  nbits;
    int32_t  bits[4];
    uint32_t op_begin;
    uint32_t op_end;
} mlb_tile_segment_t;
int  mlb_tile_plan(const mlb_op_t *ops, size_t num_ops, uint32_t num_qubits, int dtype, int fuse1q,
                   mlb_tile_pass_t *passes, size_t *num_passes, mlb_tile_segment_t *segments,
                   size_t *num_segments, mlb_op_t *planned_ops, size_t *num_planned);
/* The fused complex64 path's plan for these ops, as a flush in MLB_EXEC_FUSED
 * mode would launch it (host only).  Passes: tile = qubits 0..num_low-1 plus
 * hbits[0..num_high-1] (tile bit num_low + i <-> hbits[i]); blocks
 * [block_begin, block_begin + num_blocks) act on every tile in order.  A
 * block acts on tile bits pos[0..4] (block index bit j <-> pos[j]); rows
 * lists the other 8 tile bits.  Its operand image (16 KiB at image * 16384)
 * holds U' = [Re U -Im U; Im U Re U] as bf16 hi (first 8 KiB) and lo
 * (U' - hi) in the tensor core's K-major 128-byte-swizzled layout: element
 * (n, k) at byte (n / 8) * 1024 + (n % 8) * 128 + 2 k with the 16-byte
 * chunk index XORed with n % 8.  Call with NULL buffers to learn the sizes. */
typedef struct {
    uint8_t  hbits[12];
    uint8_t  num_low;
    uint8_t  num_high;
    uint8_t  reserved[2];
    uint64_t num_tiles;
    uint32_t block_begin;
    uint32_t num_blocks;
} mlb_fused_pass_t;
typedef struct {
    uint8_t  pos[5];
    uint8_t  rows[8];
    uint8_t  reserved[3];
    uint32_t image;
} mlb_fused_block_t;
int  mlb_fused_plan(const mlb_op_t *ops, size_t num_ops, uint32_t num_qubits,
                    mlb_fused_pass_t *passes, size_t *num_passes, mlb_fused_block_t *blocks,
                    size_t *num_blocks, void *images, size_t *image_bytes);
int  mlb_total_kernel_launches(uint64_t *out);

/* ---- batched adjoint gradient (hardware-efficient ansatz) ---------------- */
/* Energy E(theta) = <psi|H|psi> and dE/dtheta for the tape of
 * vqe_build_hea_diff_circuit (vqe.c:1946-1981): X on the set bits of
 * hf_reference, then per layer RY(q, theta[2(lN+q)]), RZ(q, theta[2(lN+q)+1])
 * for every qubit and the CNOT(q, q+1) ladder.  H = sum_k c_k P_k with P_k
 * given by its X mask (X or Y qubits) and Z mask (Z or Y qubits).  The
 * gradient equals moonlab_diff_backward_pauli_sum's (differentiable.c:478). */
typedef struct mlb_hea mlb_hea_t;
int  mlb_hea_create(uint32_t num_qubits, uint32_t num_layers, uint64_t hf_reference,
                    size_t num_terms, const uint64_t *xmasks, const uint64_t *zmasks,
                    const double *coeffs, int dtype, int device, mlb_hea_t **out);
void mlb_hea_free(mlb_hea_t *h);
int  mlb_hea_num_parameters(const mlb_hea_t *h, uint32_t *out);
/* B parameter vectors params[B][P] -> energies[B] and grads[B][P] (either may
 * be NULL).  on_device = 1: all three are device pointers. */
int  mlb_hea_evaluate(mlb_hea_t *h, size_t batch, const double *params, double *energies,
                      double *grads, int on_device);
/* Device bytes an evaluation may hold in states: psi, lambda and checkpoints
 * (0 = 80% of free device memory). */
int  mlb_hea_set_memory_budget(mlb_hea_t *h, size_t bytes);
int  mlb_hea_plan_stats(const mlb_hea_t *h, uint32_t *fwd_passes, uint32_t *lambda_passes,
                        uint32_t *bwd_passes);
/* Checkpoints: the tape runs in segments of ceil(sqrt(L)) layers; with
 * checkpoints the forward sweep keeps psi at each segment boundary and the
 * backward sweep restores it there, so the uncompute by inverse gates never
 * spans more than one segment (C - 1 extra states per vector for C
 * segments).  mode 0 (default): checkpoints when they fit beside the whole
 * batch in the budget; when memory is short they are dropped first, then the
 * batch runs in sub-batches.  mode 1: always (sub-batches if needed);
 * mode -1: never. */
int  mlb_hea_set_checkpointing(mlb_hea_t *h, int mode);
/* What the last mlb_hea_evaluate did: layers per segment, whether it kept
 * checkpoints, and how many sub-batches it ran. */
int  mlb_hea_last_eval_stats(const mlb_hea_t *h, uint32_t *segment_layers, int *checkpoints_used,
                             size_t *sub_batches);
/* complex64 problems with N >= 13: the forward sweep runs on the tensor
 * cores -- each checkpoint segment's gates grouped into <= 5-qubit blocks
 * and applied by the fused complex64 kernel, with every vector's operand
 * images built on the device from its angles.  The FP32 accumulation shrinks
 * |psi| by ~4e-7 per block, so energies and gradients are divided by the
 * forward state's squared norm (both carry it).  mode 0 (default): on for
 * complex64 when the plan exists; 1: on (MLB_ERR_NOT_SUPPORTED without a
 * plan); -1: off (the CUDA-core forward passes).  The backward sweep always
 * runs on the CUDA cores.  *fused: whether the last evaluation used it;
 * *passes, *blocks: the fused forward plan's passes and blocks (0 without a
 * plan); any output may be NULL. */
int  mlb_hea_set_fused_forward(mlb_hea_t *h, int mode);
int  mlb_hea_last_forward_fused(const mlb_hea_t *h, int *fused, uint32_t *passes, uint32_t *blocks);
/* Quantum geometry at one parameter vector (complex128 problems): the
 * Fubini-Study metric g = Re Q and the Berry curvature F = -2 Im Q of
 * Q_ij = <d_i psi|d_j psi> - <d_i psi|psi><psi|d_j psi>, each P x P
 * row-major (either may be NULL), filled as vqe_compute_qgt and
 * vqe_compute_berry_curvature fill them (src/algorithms/vqe_qng.c:166-232;
 * replaces the per-entry host loops behind moonlab_vqe_qgt /
 * moonlab_vqe_berry_curvature, src/applications/moonlab_vqe_export.c:53-86).
 * psi and the P derivative states run as one batch of P + 1 states through
 * the forward passes, and their Gram matrix comes from one FP64 kernel:
 * (P + 1) states of 2^N amplitudes must fit on the device. */
int  mlb_hea_geometry(mlb_hea_t *h, const double *params, double *metric, double *curvature);
const char *mlb_hea_last_error(void);

/* ---- error text ---------------------------------------------------------- */
const char *mlb_status_string(int status);
const char *mlb_last_error(void);   /* thread-local detail of the last failure */

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* MOONLAB_B200_H */
