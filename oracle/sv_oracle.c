/*
 * sv_oracle.c -- plain-C restatement of the reference's dense complex128
 * state-vector path (tsotchke/moonlab 1.2.0).  TEST INFRASTRUCTURE: the
 * parity checker for the CUDA engine, never part of the product path.
 *
 * Every function names the reference function and file:line whose
 * behaviour it restates.  Floating point: built with -ffp-contract=off, and
 * every accumulation that the reference's Release build (-O3
 * -ffp-contract=fast, cmake/compiler_flags.cmake:123-139) compiles to a
 * fused multiply-add is written here as an explicit fma(); the others
 * round the product and the sum separately.  Which loops fuse was read off
 * the x86-64 assembly of the reference sources built with those flags:
 *   fused:    measurement_probability_one (measurement.c:93),
 *             measurement_single_qubit's norm loop (:214),
 *             the qgtl probability dump re*re + im*im (fma(re, re, im*im)),
 *   separate: measurement_sample (:572), measurement_all_qubits (:281),
 *             measurement_correlation_zz (:522), quantum_measure
 *             (gates.c:1150-1199), quantum_measure_all_fast (gates.c:1314).
 * With that, sums and sampled outcomes match the reference bit for bit.
 * Gate arithmetic follows the reference's CPU loops algebraically; it agrees
 * with the reference library to ~1e-15 per amplitude (rounding of complex
 * products), and tests pin that.
 */
#include "sv_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

#define AMP(a) ((cplx *)(a))
#define SVO_SMALL_NORM 1e-15 /* measurement.c:32 MEASUREMENT_SMALL_NORM */

static inline int bit(uint64_t i, int q) { return (int)((i >> q) & 1u); }

/* quantum_state_init (state.c:39): |0...0>. */
void svo_init_zero(double *amp, int n)
{
    memset(amp, 0, ((size_t)1 << n) * 2 * sizeof(double));
    amp[0] = 1.0;
}

/* ------------------------------------------------------------------ */
/* single-qubit gates (gates.c:123-565)                                 */
/* ------------------------------------------------------------------ */

/* apply_single_qubit_gate (gates.c:1354): generic 2x2 on the pair
 * (i, i | 1<<t); m is the GPU-route layout of state_gpu.cu:136-151
 * (row-major, (re,im) per entry). */
void svo_apply_1q_matrix(double *amp, int n, int t, const double m[8])
{
    cplx *a = AMP(amp);
    const cplx m00 = CMPLX(m[0], m[1]), m01 = CMPLX(m[2], m[3]);
    const cplx m10 = CMPLX(m[4], m[5]), m11 = CMPLX(m[6], m[7]);
    const uint64_t stride = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t base = 0; base < dim; base += 2 * stride)
        for (uint64_t i = 0; i < stride; i++) {
            const cplx a0 = a[base + i], a1 = a[base + i + stride];
            a[base + i]          = m00 * a0 + m01 * a1;
            a[base + i + stride] = m10 * a0 + m11 * a1;
        }
}

/* gate_pauli_x (gates.c:123): swap the two halves of every block. */
static void g_x(cplx *a, int n, int t)
{
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            cplx tmp = a[b + i]; a[b + i] = a[b + i + s]; a[b + i + s] = tmp;
        }
}

/* gate_pauli_y (gates.c:155): a0' = -i a1, a1' = i a0. */
static void g_y(cplx *a, int n, int t)
{
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            const cplx a0 = a[b + i], a1 = a[b + i + s];
            a[b + i]     = CMPLX(cimag(a1), -creal(a1));
            a[b + i + s] = CMPLX(-cimag(a0), creal(a0));
        }
}

/* gate_pauli_z (gates.c:197): negate the |1> half. */
static void g_z(cplx *a, int n, int t)
{
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) a[b + i + s] = -a[b + i + s];
}

/* gate_hadamard (gates.c:226) via simd_hadamard_pair: (a0 +- a1) / sqrt 2. */
static void g_h(cplx *a, int n, int t)
{
    const double r = 0.70710678118654752440; /* QC_SQRT2_INV */
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            const cplx a0 = a[b + i], a1 = a[b + i + s];
            a[b + i]     = (a0 + a1) * r;
            a[b + i + s] = (a0 - a1) * r;
        }
}

/* qs_phase_on_one (gates.c:275) and gate_s / gate_s_dagger (:311/:345):
 * multiply the |1> half by a phase.  mode 1: +i, -1: -i, 0: generic. */
static void g_phase1(cplx *a, int n, int t, int mode, cplx ph)
{
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            const cplx v = a[b + i + s];
            if (mode == 1)       a[b + i + s] = CMPLX(-cimag(v), creal(v));
            else if (mode == -1) a[b + i + s] = CMPLX(cimag(v), -creal(v));
            else                 a[b + i + s] = v * ph;
        }
}

/* gate_rx (gates.c:385): a0' = c a0 - i s a1, a1' = c a1 - i s a0. */
static void g_rx(cplx *a, int n, int t, double theta)
{
    const double c = cos(theta / 2.0), sn = sin(theta / 2.0);
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            const cplx a0 = a[b + i], a1 = a[b + i + s];
            a[b + i]     = CMPLX(c * creal(a0) + sn * cimag(a1), c * cimag(a0) - sn * creal(a1));
            a[b + i + s] = CMPLX(c * creal(a1) + sn * cimag(a0), c * cimag(a1) - sn * creal(a0));
        }
}

/* gate_ry (gates.c:425): a0' = c a0 - s a1, a1' = s a0 + c a1. */
static void g_ry(cplx *a, int n, int t, double theta)
{
    const double c = cos(theta / 2.0), sn = sin(theta / 2.0);
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            const cplx a0 = a[b + i], a1 = a[b + i + s];
            a[b + i]     = CMPLX(c * creal(a0) - sn * creal(a1), c * cimag(a0) - sn * cimag(a1));
            a[b + i + s] = CMPLX(sn * creal(a0) + c * creal(a1), sn * cimag(a0) + c * cimag(a1));
        }
}

/* gate_rz (gates.c:481): |0> half * e^{-i theta/2}, |1> half * e^{+i theta/2}. */
static void g_rz(cplx *a, int n, int t, double theta)
{
    const cplx p0 = cexp(-I * theta / 2.0), p1 = cexp(I * theta / 2.0);
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            a[b + i] *= p0;
            a[b + i + s] *= p1;
        }
}

/* gate_u3 (gates.c:521). */
static void g_u3(cplx *a, int n, int t, double th, double phi, double lam)
{
    const double c = cos(th / 2.0), sn = sin(th / 2.0);
    const cplx ephi = cexp(I * phi), elam = cexp(I * lam), epl = cexp(I * (phi + lam));
    const uint64_t s = (uint64_t)1 << t, dim = (uint64_t)1 << n;
    for (uint64_t b = 0; b < dim; b += 2 * s)
        for (uint64_t i = 0; i < s; i++) {
            const cplx a0 = a[b + i], a1 = a[b + i + s];
            a[b + i]     = c * a0 - elam * sn * a1;
            a[b + i + s] = ephi * sn * a0 + epl * c * a1;
        }
}

/* ------------------------------------------------------------------ */
/* two- and multi-qubit gates (gates.c:571-1048)                        */
/* ------------------------------------------------------------------ */

/* apply_two_qubit_gate / qsim_gpu_route_apply_2q_matrix (state_gpu.cu:153-167):
 * 4x4 on basis |q1 q0>, q0 the low bit of the 4x4 index. */
void svo_apply_2q_matrix(double *amp, int n, int q0, int q1, const double m[32])
{
    cplx *a = AMP(amp);
    cplx M[4][4];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) M[r][c] = CMPLX(m[r * 8 + c * 2], m[r * 8 + c * 2 + 1]);
    const uint64_t dim = (uint64_t)1 << n, b0 = (uint64_t)1 << q0, b1 = (uint64_t)1 << q1;
    for (uint64_t i = 0; i < dim; i++) {
        if (i & (b0 | b1)) continue;
        const uint64_t idx[4] = { i, i | b0, i | b1, i | b0 | b1 };
        cplx v[4], w[4];
        for (int k = 0; k < 4; k++) v[k] = a[idx[k]];
        for (int r = 0; r < 4; r++) {
            w[r] = 0;
            for (int c = 0; c < 4; c++) w[r] += M[r][c] * v[c];
        }
        for (int k = 0; k < 4; k++) a[idx[k]] = w[k];
    }
}

/* gate_mcx (gates.c:980) / gate_cnot (:571) / gate_toffoli (:905):
 * swap the target pair where every control bit is 1. */
void svo_apply_mcx(double *amp, int n, uint64_t cmask, int target)
{
    cplx *a = AMP(amp);
    const uint64_t dim = (uint64_t)1 << n, tb = (uint64_t)1 << target;
    for (uint64_t i = 0; i < dim; i++)
        if ((i & cmask) == cmask && !(i & tb)) {
            cplx tmp = a[i]; a[i] = a[i | tb]; a[i | tb] = tmp;
        }
}

/* gate_mcz (gates.c:1019) / gate_cz (:641): negate where all bits set. */
void svo_apply_mcz(double *amp, int n, uint64_t mask)
{
    cplx *a = AMP(amp);
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++)
        if ((i & mask) == mask) a[i] = -a[i];
}

/* gate_cy (gates.c:670): where c=1,t=0: a_i' = -i a_j, a_j' = i a_i. */
static void g_cy(cplx *a, int n, int c, int t)
{
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++)
        if (bit(i, c) && !bit(i, t)) {
            const uint64_t j = i ^ ((uint64_t)1 << t);
            const cplx a0 = a[i], a1 = a[j];
            a[i] = CMPLX(cimag(a1), -creal(a1));
            a[j] = CMPLX(-cimag(a0), creal(a0));
        }
}

/* gate_swap (gates.c:699). */
static void g_swap(cplx *a, int n, int q1, int q2)
{
    if (q1 == q2) return;
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++)
        if (bit(i, q1) == 0 && bit(i, q2) == 1) {
            const uint64_t j = i ^ ((uint64_t)1 << q1) ^ ((uint64_t)1 << q2);
            cplx tmp = a[i]; a[i] = a[j]; a[j] = tmp;
        }
}

/* gate_cphase (gates.c:737): multiply |11> by e^{i theta}. */
static void g_cphase(cplx *a, int n, int c, int t, double theta)
{
    const cplx ph = cexp(I * theta);
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++)
        if (bit(i, c) && bit(i, t)) a[i] *= ph;
}

/* gate_crx / gate_cry (gates.c:800 / :835): the RX / RY pair update on the
 * control = 1 half. */
static void g_crxy(cplx *a, int n, int c, int t, double theta, int is_y)
{
    const double ch = cos(theta / 2.0), sh = sin(theta / 2.0);
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++)
        if (bit(i, c) && !bit(i, t)) {
            const uint64_t j = i ^ ((uint64_t)1 << t);
            const cplx a0 = a[i], a1 = a[j];
            if (is_y) {
                a[i] = CMPLX(ch * creal(a0) - sh * creal(a1), ch * cimag(a0) - sh * cimag(a1));
                a[j] = CMPLX(ch * creal(a1) + sh * creal(a0), ch * cimag(a1) + sh * cimag(a0));
            } else {
                a[i] = CMPLX(ch * creal(a0) + sh * cimag(a1), ch * cimag(a0) - sh * creal(a1));
                a[j] = CMPLX(ch * creal(a1) + sh * cimag(a0), ch * cimag(a1) - sh * creal(a0));
            }
        }
}

/* gate_crz (gates.c:870): control = 1 half gets diag(e^{-i t/2}, e^{+i t/2}). */
static void g_crz(cplx *a, int n, int c, int t, double theta)
{
    const cplx p0 = cexp(-I * theta / 2.0), p1 = cexp(I * theta / 2.0);
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++)
        if (bit(i, c)) a[i] *= bit(i, t) ? p1 : p0;
}

/* gate_fredkin (gates.c:940): swap (t1,t2) where control = 1. */
static void g_fredkin(cplx *a, int n, int c, int t1, int t2)
{
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++)
        if (bit(i, c) && bit(i, t1) == 0 && bit(i, t2) == 1) {
            const uint64_t j = i ^ ((uint64_t)1 << t1) ^ ((uint64_t)1 << t2);
            cplx tmp = a[i]; a[i] = a[j]; a[j] = tmp;
        }
}

static int valid_q(int n, int q) { return q >= 0 && q < n; }

/* apply_one_gate (moonlab_qgtl_backend.c:119-149) extended to the gates.c
 * surface.  CY follows the qgtl composition S . CNOT . S^dagger
 * (moonlab_qgtl_backend.c:138-144); ZZ(theta) follows the reference form
 * CNOT(i,j) . RZ(j, theta) . CNOT(i,j) (qaoa.c:745-753). */
int svo_apply_gate(double *amp, int n, const svo_gate_t *g)
{
    cplx *a = AMP(amp);
    const int q0 = g->q0, q1 = g->q1;
    switch (g->type) {
    case SVO_I: return 0;
    case SVO_X: if (!valid_q(n, q0)) return -1; g_x(a, n, q0); return 0;
    case SVO_Y: if (!valid_q(n, q0)) return -1; g_y(a, n, q0); return 0;
    case SVO_Z: if (!valid_q(n, q0)) return -1; g_z(a, n, q0); return 0;
    case SVO_H: if (!valid_q(n, q0)) return -1; g_h(a, n, q0); return 0;
    case SVO_S: if (!valid_q(n, q0)) return -1; g_phase1(a, n, q0, 1, 0); return 0;
    case SVO_SDG: if (!valid_q(n, q0)) return -1; g_phase1(a, n, q0, -1, 0); return 0;
    case SVO_T: if (!valid_q(n, q0)) return -1; g_phase1(a, n, q0, 0, cexp(I * M_PI / 4.0)); return 0;
    case SVO_TDG: if (!valid_q(n, q0)) return -1; g_phase1(a, n, q0, 0, cexp(-I * M_PI / 4.0)); return 0;
    case SVO_PHASE: if (!valid_q(n, q0)) return -1; g_phase1(a, n, q0, 0, cexp(I * g->theta)); return 0;
    case SVO_RX: if (!valid_q(n, q0)) return -1; g_rx(a, n, q0, g->theta); return 0;
    case SVO_RY: if (!valid_q(n, q0)) return -1; g_ry(a, n, q0, g->theta); return 0;
    case SVO_RZ: if (!valid_q(n, q0)) return -1; g_rz(a, n, q0, g->theta); return 0;
    case SVO_U3: if (!valid_q(n, q0)) return -1; g_u3(a, n, q0, g->theta, g->theta2, g->theta3); return 0;
    default: break;
    }
    if (!valid_q(n, q0) || !valid_q(n, q1)) return -1;
    if (q0 == q1) return g->type == SVO_SWAP ? 0 : -1;
    switch (g->type) {
    case SVO_CNOT: svo_apply_mcx(amp, n, (uint64_t)1 << q0, q1); return 0;
    case SVO_CZ: svo_apply_mcz(amp, n, ((uint64_t)1 << q0) | ((uint64_t)1 << q1)); return 0;
    case SVO_CY:
        g_phase1(a, n, q1, 1, 0);
        svo_apply_mcx(amp, n, (uint64_t)1 << q0, q1);
        g_phase1(a, n, q1, -1, 0);
        return 0;
    case SVO_SWAP: g_swap(a, n, q0, q1); return 0;
    case SVO_CPHASE: g_cphase(a, n, q0, q1, g->theta); return 0;
    case SVO_CRX: g_crxy(a, n, q0, q1, g->theta, 0); return 0;
    case SVO_CRY: g_crxy(a, n, q0, q1, g->theta, 1); return 0;
    case SVO_CRZ: g_crz(a, n, q0, q1, g->theta); return 0;
    case SVO_ZZ:
        svo_apply_mcx(amp, n, (uint64_t)1 << q0, q1);
        g_rz(a, n, q1, g->theta);
        svo_apply_mcx(amp, n, (uint64_t)1 << q0, q1);
        return 0;
    case SVO_TOFFOLI:
        if (!valid_q(n, g->q2) || g->q2 == q0 || g->q2 == q1) return -1;
        svo_apply_mcx(amp, n, ((uint64_t)1 << q0) | ((uint64_t)1 << q1), g->q2);
        return 0;
    case SVO_FREDKIN:
        if (!valid_q(n, g->q2) || g->q2 == q0 || g->q2 == q1) return -1;
        g_fredkin(a, n, q0, q1, g->q2);
        return 0;
    default: return -2;
    }
}

int svo_apply_circuit(double *amp, int n, const svo_gate_t *gates, size_t num_gates)
{
    for (size_t i = 0; i < num_gates; i++) {
        int rc = svo_apply_gate(amp, n, &gates[i]);
        if (rc) return rc;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* reductions (measurement.c:73-540)                                   */
/* ------------------------------------------------------------------ */

/* measurement_probability_one (measurement.c:73): sum cabs^2 over bit q set,
 * in index order. */
double svo_probability_one(const double *amp, int n, int q)
{
    const cplx *a = (const cplx *)amp;
    const uint64_t dim = (uint64_t)1 << n, mask = (uint64_t)1 << q;
    double p = 0.0;
    for (uint64_t i = 0; i < dim; i++)
        if (i & mask) { const double h = cabs(a[i]); p = fma(h, h, p); }
    return p;
}

/* measurement_probability_distribution (measurement.c:140): cabs(a)^2. */
void svo_probability_distribution(const double *amp, int n, double *out)
{
    const cplx *a = (const cplx *)amp;
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++) { const double h = cabs(a[i]); out[i] = h * h; }
}

/* moonlab_qgtl_execute probability dump (moonlab_qgtl_backend.c:199-210):
 * re*re + im*im. */
void svo_qgtl_probabilities(const double *amp, int n, double *out)
{
    const uint64_t dim = (uint64_t)1 << n;
    for (uint64_t i = 0; i < dim; i++) {
        const double re = amp[2 * i], im = amp[2 * i + 1];
        out[i] = fma(re, re, im * im);
    }
}

/* measurement_expectation_z (measurement.c:428) = 1 - 2 P1. */
double svo_expectation_z(const double *amp, int n, int q)
{
    return 1.0 - 2.0 * svo_probability_one(amp, n, q);
}

/* measurement_expectation_x (measurement.c:442). */
double svo_expectation_x(const double *amp, int n, int q)
{
    const cplx *a = (const cplx *)amp;
    const uint64_t dim = (uint64_t)1 << n, mask = (uint64_t)1 << q;
    double e = 0.0;
    for (uint64_t i = 0; i < dim; i++) {
        const uint64_t j = i ^ mask;
        if (j > i) e += creal(conj(a[i]) * a[j] + conj(a[j]) * a[i]);
    }
    return e;
}

/* measurement_expectation_y (measurement.c:473). */
double svo_expectation_y(const double *amp, int n, int q)
{
    const cplx *a = (const cplx *)amp;
    const uint64_t dim = (uint64_t)1 << n, mask = (uint64_t)1 << q;
    double e = 0.0;
    for (uint64_t i = 0; i < dim; i++) {
        const uint64_t j = i ^ mask;
        if (j > i) {
            const double f = (i & mask) ? -1.0 : 1.0;
            e += f * cimag(conj(a[i]) * a[j] - conj(a[j]) * a[i]);
        }
    }
    return e;
}

/* measurement_correlation_zz (measurement.c:509). */
double svo_correlation_zz(const double *amp, int n, int q1, int q2)
{
    const cplx *a = (const cplx *)amp;
    const uint64_t dim = (uint64_t)1 << n, m1 = (uint64_t)1 << q1, m2 = (uint64_t)1 << q2;
    double p00 = 0, p01 = 0, p10 = 0, p11 = 0;
    for (uint64_t i = 0; i < dim; i++) {
        const double h = cabs(a[i]), p = h * h;
        const int b1 = (i & m1) != 0, b2 = (i & m2) != 0;
        if (!b1 && !b2) p00 += p; else if (!b1 && b2) p01 += p; else if (b1 && !b2) p10 += p; else p11 += p;
    }
    return p00 + p11 - p01 - p10;
}

/* quantum_state_normalize / is_normalized norm (state.c:206-254): sum |a|^2. */
double svo_norm_sq(const double *amp, int n)
{
    const uint64_t dim = (uint64_t)1 << n;
    double s = 0.0;
    for (uint64_t i = 0; i < dim; i++) s += amp[2 * i] * amp[2 * i] + amp[2 * i + 1] * amp[2 * i + 1];
    return s;
}

/* <psi|P|psi> for the Pauli string with X-part xmask and Z-part zmask
 * (Y on a qubit = both bits): the value moonlab_diff_expect_pauli_sum
 * (differentiable.c:408) forms per term as Re<psi|P psi> after applying the
 * gate_pauli_* factors (apply_pauli_string, differentiable.c:395).  Computed
 * here by the same route: clone, apply factors in qubit order, inner product. */
double svo_expect_pauli_string(const double *amp, int n, uint64_t xmask, uint64_t zmask)
{
    const uint64_t dim = (uint64_t)1 << n;
    cplx *s = malloc(dim * sizeof(cplx));
    if (!s) return NAN;
    memcpy(s, amp, dim * sizeof(cplx));
    for (int q = 0; q < n; q++) {
        const int x = (xmask >> q) & 1, z = (zmask >> q) & 1;
        if (x && z) g_y(s, n, q);
        else if (x) g_x(s, n, q);
        else if (z) g_z(s, n, q);
    }
    const cplx *a = (const cplx *)amp;
    cplx acc = 0;
    for (uint64_t i = 0; i < dim; i++) acc += conj(a[i]) * s[i];
    free(s);
    return creal(acc);
}

/* ------------------------------------------------------------------ */
/* sampling and collapse                                               */
/* ------------------------------------------------------------------ */

/* measurement_sample (measurement.c:551-601): sequential FP64 CDF of
 * cabs(a)^2, then per uniform the first index with cdf >= u (binary search
 * clamped to dim-1). */
void svo_measurement_sample(const double *amp, int n, uint64_t *outcomes,
                            int num_samples, const double *u)
{
    const cplx *a = (const cplx *)amp;
    const uint64_t dim = (uint64_t)1 << n;
    double *cdf = malloc(dim * sizeof(double));
    if (!cdf) { for (int s = 0; s < num_samples; s++) outcomes[s] = 0; return; }
    double cum = 0.0;
    for (uint64_t i = 0; i < dim; i++) { const double h = cabs(a[i]); const double p = h * h; cum += p; cdf[i] = cum; }
    for (int s = 0; s < num_samples; s++) {
        uint64_t lo = 0, hi = dim - 1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) / 2;
            if (cdf[mid] < u[s]) lo = mid + 1; else hi = mid;
        }
        outcomes[s] = lo;
    }
    free(cdf);
}

/* measurement_all_qubits outcome rule (measurement.c:263-307) and
 * quantum_measure_all_fast (gates.c:1293): first i with u < cum_i, else the
 * last index with nonzero probability, else 0. */
uint64_t svo_measure_all_index(const double *amp, int n, double u)
{
    const cplx *a = (const cplx *)amp;
    const uint64_t dim = (uint64_t)1 << n;
    double cum = 0.0;
    uint64_t last_nz = 0;
    int have_nz = 0;
    for (uint64_t i = 0; i < dim; i++) {
        const double h = cabs(a[i]);
        const double p = h * h;
        if (p > 0.0) { last_nz = i; have_nz = 1; }
        cum += p;
        if (u < cum) return i;
    }
    return have_nz ? last_nz : 0;
}

/* collapse to a basis state (measurement.c:300-303). */
void svo_collapse_to_index(double *amp, int n, uint64_t idx)
{
    svo_init_zero(amp, n);
    amp[0] = 0.0;
    amp[2 * idx] = 1.0;
}

/* measurement_single_qubit (measurement.c:181-241): outcome 1 iff u < P1;
 * zero the other half, renormalise by 1/sqrt(norm) (norm = sum cabs^2 of the
 * kept half in index order); -1 when the kept norm <= 1e-15. */
int svo_measurement_single_qubit(double *amp, int n, int q, double u)
{
    cplx *a = AMP(amp);
    const uint64_t dim = (uint64_t)1 << n, mask = (uint64_t)1 << q;
    const double p1 = svo_probability_one(amp, n, q);
    const int r = (u < p1) ? 1 : 0;
    double nf = 0.0;
    for (uint64_t i = 0; i < dim; i++) {
        if (((i & mask) ? 1 : 0) != r) a[i] = 0.0;
        else { const double h = cabs(a[i]); nf = fma(h, h, nf); }
    }
    if (nf <= SVO_SMALL_NORM) return -1;
    const double inv = 1.0 / sqrt(nf);
    for (uint64_t i = 0; i < dim; i++) a[i] *= inv;
    return r;
}

/* quantum_measure, computational basis (gates.c:1117-1241): P0 summed
 * block by block (lower halves in order), outcome 0 iff u < P0, kept-half
 * norm summed block by block, divide by sqrt(norm).  Returns -1 (state
 * untouched past the zeroing) when the kept norm <= 1e-15, as the
 * reference returns its zero result there. */
int svo_quantum_measure(double *amp, int n, int q, double u, double *prob_out)
{
    cplx *a = AMP(amp);
    const uint64_t s = (uint64_t)1 << q, dim = (uint64_t)1 << n;
    double p0 = 0.0, p1 = 0.0;
    for (uint64_t b = 0; b < dim; b += 2 * s) {
        for (uint64_t i = 0; i < s; i++) { const double m = cabs(a[b + i]); p0 += m * m; }
        for (uint64_t i = 0; i < s; i++) { const double m = cabs(a[b + s + i]); p1 += m * m; }
    }
    const int r = (u < p0) ? 0 : 1;
    if (prob_out) *prob_out = r == 0 ? p0 : p1;
    double nrm = 0.0;
    for (uint64_t b = 0; b < dim; b += 2 * s) {
        const uint64_t keep = r == 0 ? b : b + s, drop = r == 0 ? b + s : b;
        memset(&a[drop], 0, s * sizeof(cplx));
        for (uint64_t i = 0; i < s; i++) { const double m = cabs(a[keep + i]); nrm += m * m; }
    }
    if (nrm <= 1e-15) return -1;
    nrm = sqrt(nrm);
    for (uint64_t i = 0; i < dim; i++) a[i] /= nrm;
    return r;
}

/* ------------------------------------------------------------------ */
/* circuit execution and the simulator backend                          */
/* ------------------------------------------------------------------ */

/* xorshift64_step (moonlab_qgtl_backend.c:159-167). */
uint64_t svo_xorshift64(uint64_t *s)
{
    uint64_t x = *s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *s = x;
    return x;
}

/* splitmix64 finalizer form used for worker seeds (scheduler.c:143-149). */
uint64_t svo_splitmix64_finalizer(uint64_t x)
{
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d49bb133111ebbULL;
    return x ^ (x >> 31);
}

/* moonlab_qgtl_execute (moonlab_qgtl_backend.c:169-247): gate walk from
 * |0..0>, optional re^2+im^2 probability dump, and per shot a fresh
 * xorshift64 draw u = (r >> 11) 2^-53 fed to measurement_all_qubits on a
 * clone of the final state (the clone makes every shot see the same
 * distribution, so the rule is applied to the unchanged state here).
 * rng_seed must be nonzero (0 means a clock seed in the reference). */
int svo_qgtl_execute(int n, const svo_gate_t *gates, size_t num_gates,
                     int num_shots, uint64_t rng_seed,
                     uint64_t *outcomes, double *probabilities)
{
    const uint64_t dim = (uint64_t)1 << n;
    double *amp = malloc(dim * 2 * sizeof(double));
    if (!amp) return -302;
    svo_init_zero(amp, n);
    if (svo_apply_circuit(amp, n, gates, num_gates)) { free(amp); return -304; }
    if (probabilities) svo_qgtl_probabilities(amp, n, probabilities);
    uint64_t seed = rng_seed;
    for (int s = 0; s < num_shots; s++) {
        const uint64_t r = svo_xorshift64(&seed);
        const double u = (double)(r >> 11) / (double)(1ULL << 53);
        outcomes[s] = svo_measure_all_index(amp, n, u);
    }
    free(amp);
    return 0;
}

/* simulator_backend_execute (scheduler.c:194-239): worker w runs shots
 * [w*S/W, (w+1)*S/W) through moonlab_qgtl_execute seeded with
 * splitmix64(seed ^ (w << 32)).  Workers capped at the shot count. */
int svo_scheduler_simulator(int n, const svo_gate_t *gates, size_t num_gates,
                            int total_shots, int num_workers, uint64_t rng_seed,
                            uint64_t *outcomes)
{
    if (total_shots <= 0) return -501;
    if (num_workers > total_shots) num_workers = total_shots;
    if (num_workers < 1) num_workers = 1;
    for (int w = 0; w < num_workers; w++) {
        const int start = (int)((long long)w * total_shots / num_workers);
        const int end = (int)((long long)(w + 1) * total_shots / num_workers);
        if (end <= start) continue;
        const uint64_t seed = svo_splitmix64_finalizer(rng_seed ^ ((uint64_t)w << 32));
        int rc = svo_qgtl_execute(n, gates, num_gates, end - start, seed, outcomes + start, NULL);
        if (rc) return -503;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* HEA adjoint gradient                                                */
/* ------------------------------------------------------------------ */

typedef struct { int kind; int q0, q1; double theta; long pidx; } hop_t; /* 0 X, 1 RY, 2 RZ, 3 CNOT */

static void hop_apply(cplx *a, int n, const hop_t *o, double sign)
{
    switch (o->kind) {
    case 0: g_x(a, n, o->q0); break;
    case 1: g_ry(a, n, o->q0, sign * o->theta); break;
    case 2: g_rz(a, n, o->q0, sign * o->theta); break;
    case 3: svo_apply_mcx((double *)a, n, (uint64_t)1 << o->q0, o->q1); break;
    }
}

static void pauli_apply(cplx *a, int n, const char *ps)
{
    for (int q = 0; q < n; q++) {
        const char c = ps[q];
        if (c == 'X' || c == 'x') g_x(a, n, q);
        else if (c == 'Y' || c == 'y') g_y(a, n, q);
        else if (c == 'Z' || c == 'z') g_z(a, n, q);
    }
}

/* vqe_compute_gradient_adjoint (vqe.c:1986) on the HEA tape built by
 * vqe_build_hea_diff_circuit (vqe.c:1946-1981): X on hf bits, then per
 * layer RY(p[2(l n + q)]), RZ(p[2(l n + q) + 1]) per qubit and the
 * CNOT(q, q+1) ladder.  Gradient by moonlab_diff_backward_pauli_sum
 * (differentiable.c:478): per term, eta = P_k psi, walk ops in reverse,
 * grad[p] += c_k Im<eta|G|xi> (eta_G_xi, differentiable.c:295; G = Y for
 * RY, Z for RZ), then undo the op on xi and eta.  Energy as
 * moonlab_diff_expect_pauli_sum (differentiable.c:408). */
int svo_hea_energy_and_gradient(int n, int layers, uint64_t hf_reference,
                                const double *params,
                                size_t num_terms, const double *coeffs,
                                const char *paulis,
                                double *energy_out, double *grad_out)
{
    const size_t nops_max = (size_t)n + (size_t)layers * (3 * (size_t)n);
    hop_t *ops = malloc(nops_max * sizeof(hop_t));
    if (!ops) return -1;
    size_t no = 0, p = 0;
    for (int q = 0; q < n; q++)
        if (hf_reference & ((uint64_t)1 << q)) ops[no++] = (hop_t){ 0, q, -1, 0.0, -1 };
    for (int l = 0; l < layers; l++) {
        for (int q = 0; q < n; q++) {
            ops[no++] = (hop_t){ 1, q, -1, params[p], (long)p }; p++;
            ops[no++] = (hop_t){ 2, q, -1, params[p], (long)p }; p++;
        }
        for (int q = 0; q + 1 < n; q++) ops[no++] = (hop_t){ 3, q, q + 1, 0.0, -1 };
    }
    const size_t np = p;
    const uint64_t dim = (uint64_t)1 << n;
    cplx *psi = malloc(dim * sizeof(cplx)), *xi = malloc(dim * sizeof(cplx));
    cplx *eta = malloc(dim * sizeof(cplx)), *scr = malloc(dim * sizeof(cplx));
    if (!psi || !xi || !eta || !scr) { free(ops); free(psi); free(xi); free(eta); free(scr); return -2; }
    svo_init_zero((double *)psi, n);
    for (size_t i = 0; i < no; i++) hop_apply(psi, n, &ops[i], 1.0);

    if (energy_out) {
        double e = 0.0;
        for (size_t k = 0; k < num_terms; k++) {
            memcpy(scr, psi, dim * sizeof(cplx));
            pauli_apply(scr, n, paulis + k * (size_t)n);
            cplx ip = 0;
            for (uint64_t i = 0; i < dim; i++) ip += conj(psi[i]) * scr[i];
            e += coeffs[k] * creal(ip);
        }
        *energy_out = e;
    }
    if (grad_out) {
        for (size_t i = 0; i < np; i++) grad_out[i] = 0.0;
        for (size_t k = 0; k < num_terms; k++) {
            memcpy(xi, psi, dim * sizeof(cplx));
            memcpy(eta, psi, dim * sizeof(cplx));
            pauli_apply(eta, n, paulis + k * (size_t)n);
            for (size_t idx = no; idx > 0; idx--) {
                const hop_t *o = &ops[idx - 1];
                if (o->pidx >= 0) {
                    memcpy(scr, xi, dim * sizeof(cplx));
                    if (o->kind == 1) g_y(scr, n, o->q0); else g_z(scr, n, o->q0);
                    cplx v = 0;
                    for (uint64_t i = 0; i < dim; i++) v += conj(eta[i]) * scr[i];
                    grad_out[o->pidx] += coeffs[k] * cimag(v);
                }
                hop_apply(xi, n, o, -1.0);
                hop_apply(eta, n, o, -1.0);
            }
        }
    }
    free(ops); free(psi); free(xi); free(eta); free(scr);
    return 0;
}
