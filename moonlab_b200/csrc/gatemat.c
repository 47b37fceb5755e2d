/*
 * gatemat.c -- gate matrices in the GPU-route layout (8 doubles for a 2x2,
 * row-major (re, im) pairs), built with the same C99 complex expressions
 * and host libm calls (cos, sin, cexp) that the reference's gate_* functions
 * evaluate before they call qsim_gpu_route_apply_1q_matrix
 * (src/quantum/gates.c:155-565).  Compiled as C so that cexp and complex
 * arithmetic are the C library's, making every matrix entry bit-identical
 * to the reference's.
 */
#include <complex.h>
#include <math.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* gate_rx (gates.c:385-398): [[c, -is], [-is, c]] */
void mlb_mat_rx(double theta, double m[8])
{
    const double c = cos(theta / 2.0), s = sin(theta / 2.0);
    m[0] = c;   m[1] = 0.0; m[2] = 0.0; m[3] = -s;
    m[4] = 0.0; m[5] = -s;  m[6] = c;   m[7] = 0.0;
}

/* gate_ry (gates.c:436-442): [[c, -s], [s, c]] */
void mlb_mat_ry(double theta, double m[8])
{
    const double c = cos(theta / 2.0), s = sin(theta / 2.0);
    m[0] = c; m[1] = 0.0; m[2] = -s; m[3] = 0.0;
    m[4] = s; m[5] = 0.0; m[6] = c;  m[7] = 0.0;
}

/* gate_rz (gates.c:488-497): diag(cexp(-i theta/2), cexp(+i theta/2)) */
void mlb_mat_rz(double theta, double m[8])
{
    const double complex p0 = cexp(-I * theta / 2.0);
    const double complex p1 = cexp(+I * theta / 2.0);
    m[0] = creal(p0); m[1] = cimag(p0); m[2] = 0.0; m[3] = 0.0;
    m[4] = 0.0; m[5] = 0.0; m[6] = creal(p1); m[7] = cimag(p1);
}

/* qs_phase_on_one via gate_t / gate_t_dagger / gate_phase (gates.c:275-380):
 * diag(1, cexp(i phi)); which = 0: T (phi = pi/4), 1: Tdg, 2: phase(theta). */
void mlb_mat_phase1(int which, double theta, double m[8])
{
    double complex ph;
    if (which == 0) ph = cexp(I * M_PI / 4.0);
    else if (which == 1) ph = cexp(-I * M_PI / 4.0);
    else ph = cexp(I * theta);
    m[0] = 1.0; m[1] = 0.0; m[2] = 0.0; m[3] = 0.0;
    m[4] = 0.0; m[5] = 0.0; m[6] = creal(ph); m[7] = cimag(ph);
}

/* gate_u3 (gates.c:521-545). */
void mlb_mat_u3(double theta, double phi, double lambda, double m[8])
{
    const double cos_half = cos(theta / 2.0);
    const double sin_half = sin(theta / 2.0);
    const double complex e_phi = cexp(I * phi);
    const double complex e_lambda = cexp(I * lambda);
    const double complex e_phi_lambda = cexp(I * (phi + lambda));
    const double complex m01 = -e_lambda * sin_half;
    const double complex m10 = e_phi * sin_half;
    const double complex m11 = e_phi_lambda * cos_half;
    m[0] = cos_half;   m[1] = 0.0;        m[2] = creal(m01); m[3] = cimag(m01);
    m[4] = creal(m10); m[5] = cimag(m10); m[6] = creal(m11); m[7] = cimag(m11);
}

/* gate_cphase (gates.c:743): cexp(i theta) on |11>. */
void mlb_mat_cphase(double theta, double out[2])
{
    const double complex ph = cexp(I * theta);
    out[0] = creal(ph);
    out[1] = cimag(ph);
}

/* gate_crz GPU route (gates.c:880-887): RZ built from cos/sin of -+theta/2. */
void mlb_mat_crz_inner(double theta, double m[8])
{
    const double cn = cos(-theta / 2.0), sn = sin(-theta / 2.0);
    const double cp = cos(theta / 2.0), sp = sin(theta / 2.0);
    m[0] = cn; m[1] = sn; m[2] = 0.0; m[3] = 0.0;
    m[4] = 0.0; m[5] = 0.0; m[6] = cp; m[7] = sp;
}

/* ZZ(theta) = CNOT(i,j) RZ(j,theta) CNOT(i,j) (qaoa.c:745-753): the RZ phases
 * keyed on the parity of the two bits. out = {even re, even im, odd re, odd im}. */
void mlb_mat_zz(double theta, double out[4])
{
    const double complex p0 = cexp(-I * theta / 2.0);
    const double complex p1 = cexp(+I * theta / 2.0);
    out[0] = creal(p0); out[1] = cimag(p0);
    out[2] = creal(p1); out[3] = cimag(p1);
}
