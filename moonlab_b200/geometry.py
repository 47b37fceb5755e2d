"""Quantum geometry of the hardware-efficient ansatz: the quantum geometric
tensor Q_ij = <d_i psi|d_j psi> - <d_i psi|psi><psi|d_j psi>, its real part
(the Fubini-Study metric of quantum natural gradient) and its curvature part
F = -2 Im Q, and the natural-gradient direction (g + lambda I)^-1 grad.

Reference: src/algorithms/vqe_qng.c:60-99 (exact derivatives by generator
insertion: the Pauli generator right after the parameter's rotation, times
-i/2), :166-196 (vqe_compute_qgt), :198-232 (vqe_compute_berry_curvature),
:236-282 (spd_solve, vqe_natural_gradient_direction);
src/applications/moonlab_vqe_export.c:53-100 (the stable verbs).

A rotation R(t) = exp(-i t G / 2) satisfies G R(t) = i R(t + pi), so the
reference's derivative state d_i psi = (-i/2) U_after G_i U_upto |hf> is
(1/2) psi(theta + pi e_i).  The engine runs psi and the P shifted states as
one batch of P + 1 parameter vectors through the adjoint's forward passes
and forms every inner product with one FP64 Gram kernel (mlb_hea_geometry),
where the reference replays P circuits and loops over 2^n amplitudes per
tensor entry on the host.
"""
from __future__ import annotations

import math

import numpy as np

from .circuits import GATE_DTYPE

GATE_X, GATE_Y, GATE_Z, GATE_RY, GATE_RZ, GATE_CNOT = 1, 2, 3, 8, 9, 10


def hea_gates(n: int, layers: int, params, hf_reference: int = 0, insert: int | None = None) -> np.ndarray:
    """Gate records of the ansatz on |0..0>: X on the set bits of
    hf_reference, then the layers.  With insert = i, the generator of
    parameter i (Y after its RY, Z after its RZ) follows that rotation."""
    params = np.asarray(params, dtype=np.float64)
    if params.size != 2 * n * layers:
        raise ValueError(f"expected {2 * n * layers} parameters, got {params.size}")
    recs = [(GATE_X, q, -1, 0, 0.0) for q in range(n) if hf_reference >> q & 1]
    p = 0
    for _ in range(layers):
        for q in range(n):
            recs.append((GATE_RY, q, -1, 0, float(params[p])))
            if p == insert:
                recs.append((GATE_Y, q, -1, 0, 0.0))
            p += 1
            recs.append((GATE_RZ, q, -1, 0, float(params[p])))
            if p == insert:
                recs.append((GATE_Z, q, -1, 0, 0.0))
            p += 1
        recs += [(GATE_CNOT, q + 1, q, 0, 0.0) for q in range(n - 1)]
    return np.array(recs, dtype=GATE_DTYPE)


def shifted_parameters(params) -> np.ndarray:
    """The batch the engine runs: row 0 = theta, row i + 1 = theta + pi e_i
    (d_i psi = psi(row i + 1) / 2)."""
    th = np.asarray(params, dtype=np.float64).reshape(-1)
    B = np.repeat(th[None, :], th.size + 1, axis=0)
    B[1 + np.arange(th.size), np.arange(th.size)] += math.pi
    return B


def geometry(n: int, layers: int, params, hf_reference: int = 0, device: int = 0):
    """(metric, curvature), each P x P, on the device (complex128)."""
    from .vqe import HEAProblem
    prob = HEAProblem(n, layers, [], xmasks=[], zmasks=[], hf_reference=hf_reference, device=device)
    try:
        return prob.geometry(params)
    finally:
        prob.close()


def metric(n: int, layers: int, params, hf_reference: int = 0, device: int = 0) -> np.ndarray:
    """g = Re Q (vqe_compute_qgt), P x P, symmetric."""
    return geometry(n, layers, params, hf_reference, device)[0]


def berry_curvature(n: int, layers: int, params, hf_reference: int = 0, device: int = 0) -> np.ndarray:
    """F = -2 Im Q (vqe_compute_berry_curvature), P x P, antisymmetric."""
    return geometry(n, layers, params, hf_reference, device)[1]


def natural_gradient_direction(g: np.ndarray, gradient, regularization: float):
    """(g + regularization I)^-1 gradient by the reference's Gaussian
    elimination with partial pivoting (spd_solve, vqe_qng.c:236-266).  A
    pivot below 1e-300 makes the system singular: returns None, where the
    reference returns -1 and its caller falls back to the plain gradient."""
    A = np.array(g, dtype=np.float64, copy=True)
    n = A.shape[0]
    A[np.diag_indices(n)] += regularization
    w = np.array(gradient, dtype=np.float64, copy=True)
    for col in range(n):
        piv = col + int(np.argmax(np.abs(A[col:, col])))
        if abs(A[piv, col]) < 1e-300:
            return None
        if piv != col:
            A[[col, piv]] = A[[piv, col]]
            w[[col, piv]] = w[[piv, col]]
        d = A[col, col]
        for r in range(col + 1, n):
            f = A[r, col] / d
            if f == 0.0:
                continue
            A[r, col:] -= f * A[col, col:]
            w[r] -= f * w[col]
    x = np.zeros(n)
    for i in range(n - 1, -1, -1):
        s = w[i]
        for c in range(i + 1, n):
            s -= A[i, c] * x[c]
        x[i] = s / A[i, i]
    return x
