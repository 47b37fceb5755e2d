/*
 * sv_oracle.h -- CPU restatement of the reference (tsotchke/moonlab 1.2.0)
 * dense complex128 state-vector path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA engine: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.  The product path (libmoonlab_b200.so) never links,
 * loads or calls it.
 *
 * State layout matches quantum_state_t.amplitudes (src/quantum/state.h:102-131):
 * 2^n interleaved (re, im) doubles, qubit 0 = least-significant index bit.
 *
 * Pinning: tests/test_oracle_pin.py checks every function here against the
 * reference's own library built from its sources (oracle/Makefile ->
 * oracle/_ref/liboracle.so) on the reference's circuit corpus
 * (tests/oracle/corpus/circuit_corpus.json) and on seeded random states,
 * and against committed golden fixtures (tests/golden/) generated from it.
 */
#ifndef SV_ORACLE_H
#define SV_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- gate records (mirrors moonlab_qgtl_gate_t, moonlab_qgtl_backend.h:57-72,
 *      extended with the gates.c set the engine also covers) ---- */
enum {
    SVO_I = 0, SVO_X = 1, SVO_Y = 2, SVO_Z = 3, SVO_H = 4, SVO_S = 5, SVO_T = 6,
    SVO_RX = 7, SVO_RY = 8, SVO_RZ = 9, SVO_CNOT = 10, SVO_CY = 11, SVO_CZ = 12,
    SVO_SWAP = 13,
    /* beyond the QGTL enum: the rest of the gates.c surface */
    SVO_SDG = 20, SVO_TDG = 21, SVO_PHASE = 22, SVO_CPHASE = 23, SVO_CRX = 24,
    SVO_CRY = 25, SVO_CRZ = 26, SVO_ZZ = 27, SVO_TOFFOLI = 28, SVO_FREDKIN = 29,
    SVO_U3 = 30
};

typedef struct {
    int32_t type;
    int32_t q0;      /* target (1q), control for controlled 2q, qubit1 for SWAP */
    int32_t q1;      /* target for controlled 2q, qubit2 for SWAP, -1 otherwise */
    int32_t q2;      /* third qubit (Toffoli target / Fredkin t2), -1 otherwise */
    double  theta;   /* angle (phi for U3 in theta2, lambda in theta3) */
    double  theta2;
    double  theta3;
} svo_gate_t;

void     svo_init_zero(double *amp, int n);
int      svo_apply_gate(double *amp, int n, const svo_gate_t *g);
int      svo_apply_circuit(double *amp, int n, const svo_gate_t *gates, size_t num_gates);
void     svo_apply_1q_matrix(double *amp, int n, int t, const double m[8]);
void     svo_apply_2q_matrix(double *amp, int n, int q0, int q1, const double m[32]);
void     svo_apply_mcx(double *amp, int n, uint64_t control_mask, int target);
void     svo_apply_mcz(double *amp, int n, uint64_t all_mask);

double   svo_probability_one(const double *amp, int n, int q);
void     svo_probability_distribution(const double *amp, int n, double *out);
void     svo_qgtl_probabilities(const double *amp, int n, double *out);
double   svo_expectation_z(const double *amp, int n, int q);
double   svo_expectation_x(const double *amp, int n, int q);
double   svo_expectation_y(const double *amp, int n, int q);
double   svo_correlation_zz(const double *amp, int n, int q1, int q2);
double   svo_norm_sq(const double *amp, int n);
double   svo_expect_pauli_string(const double *amp, int n, uint64_t xmask, uint64_t zmask);

void     svo_measurement_sample(const double *amp, int n, uint64_t *outcomes,
                                int num_samples, const double *uniforms);
uint64_t svo_measure_all_index(const double *amp, int n, double u);
int      svo_measurement_single_qubit(double *amp, int n, int q, double u);
int      svo_quantum_measure(double *amp, int n, int q, double u, double *prob_out);
void     svo_collapse_to_index(double *amp, int n, uint64_t idx);

uint64_t svo_xorshift64(uint64_t *s);
uint64_t svo_splitmix64_finalizer(uint64_t x);
int      svo_qgtl_execute(int n, const svo_gate_t *gates, size_t num_gates,
                          int num_shots, uint64_t rng_seed,
                          uint64_t *outcomes, double *probabilities);
int      svo_scheduler_simulator(int n, const svo_gate_t *gates, size_t num_gates,
                                 int total_shots, int num_workers, uint64_t rng_seed,
                                 uint64_t *outcomes);

/* HEA adjoint gradient (vqe.c:1946-2031 + differentiable.c:438-491).
 * terms: num_terms Pauli strings, paulis[k*n + q] in {'I','X','Y','Z'}. */
int      svo_hea_energy_and_gradient(int n, int layers, uint64_t hf_reference,
                                     const double *params,
                                     size_t num_terms, const double *coeffs,
                                     const char *paulis,
                                     double *energy_out, double *grad_out);

#ifdef __cplusplus
}
#endif
#endif
