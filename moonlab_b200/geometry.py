"""Quantum geometry of the hardware-efficient ansatz: the quantum geometric
tensor Q_ij = <d_i psi|d_j psi> - <d_i psi|psi><psi|d_j psi>, its real part
(the Fubini-Study metric of quantum natural gradient) and its curvature part
F = -2 Im Q, and the natural-gradient direction (g + lambda I)^-1 grad.

Reference: src/algorithms/vqe_qng.c:42-58 (the trial state from the
Hartree-Fock bits), :60-99 (exact derivatives by generator insertion: the
Pauli generator right after the parameter's rotation, times -i/2),
:101-164 (psi, the derivatives and <psi|d_i psi>), :166-196
(vqe_compute_qgt), :198-232 (vqe_compute_berry_curvature), :270-282
(vqe_natural_gradient_direction); src/applications/moonlab_vqe_export.c:53-90
(moonlab_vqe_qgt, moonlab_vqe_berry_curvature).  The ansatz is
vqe_apply_hardware_efficient_ansatz: per layer RY(q, theta_p) and
RZ(q, theta_p+1) on every qubit, then CNOT(q, q+1) down the register.

The P derivative states are P circuit runs of the engine on the device, kept
as the rows of one P x 2^n device matrix, and Q comes from one Hermitian
Gram product of that matrix (a library GEMM) -- where the reference forms
every entry with its own loop over 2^n amplitudes on the host.
"""
from __future__ import annotations

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


class EngineRunner:
    """Runs gate records on one complex128 engine state on `device` and
    returns the output state as a device tensor (a copy)."""

    def __init__(self, n: int, device: int = 0):
        import torch
        from .statevector import StateVector
        self.sv = StateVector(n, "c128", device=device)
        self.view = torch.as_tensor(_DeviceView(self.sv.device_ptr(), 1 << n), device=f"cuda:{device}")

    def __call__(self, gates):
        self.sv.reset()
        self.sv.run(gates)
        self.sv.synchronize()
        return self.view.clone()

    def close(self) -> None:
        self.sv.close()


class _DeviceView:
    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<c16", "data": (ptr, False),
                                         "version": 3, "strides": None}


def state_and_derivatives(n: int, layers: int, params, run, hf_reference: int = 0):
    """psi (2^n), D (P x 2^n, row i = d_i psi = -i/2 U_after P_i U_upto |HF>)
    and ov (P, <psi|d_i psi>) as tensors on the runner's device."""
    import torch
    P = 2 * n * layers
    psi = run(hea_gates(n, layers, params, hf_reference))
    D = torch.empty((P, psi.numel()), dtype=torch.complex128, device=psi.device)
    for i in range(P):
        D[i] = run(hea_gates(n, layers, params, hf_reference, insert=i))
    D *= -0.5j
    ov = D @ psi.conj()  # <psi|d_i psi>
    return psi, D, ov


def geometric_tensor(n: int, layers: int, params, run, hf_reference: int = 0):
    """Q (P x P complex, Hermitian up to rounding) as a device tensor."""
    _, D, ov = state_and_derivatives(n, layers, params, run, hf_reference)
    A = D.conj() @ D.T  # <d_i psi|d_j psi>
    return A - torch_outer(ov.conj(), ov)


def torch_outer(a, b):
    return a[:, None] * b[None, :]


def _mirror_upper(M, antisymmetric: bool):
    """Upper triangle kept, lower filled from it, as the reference fills both
    halves from one computed entry (exact (anti)symmetry)."""
    import torch
    up = torch.triu(M, diagonal=0 if not antisymmetric else 1)
    return up - up.T if antisymmetric else up + torch.triu(M, diagonal=1).T


def metric(n: int, layers: int, params, run, hf_reference: int = 0) -> np.ndarray:
    """g = Re Q (vqe_compute_qgt), P x P, symmetric."""
    Q = geometric_tensor(n, layers, params, run, hf_reference)
    return _mirror_upper(Q.real, False).cpu().numpy()


def berry_curvature(n: int, layers: int, params, run, hf_reference: int = 0) -> np.ndarray:
    """F = -2 Im Q (vqe_compute_berry_curvature), P x P, antisymmetric."""
    Q = geometric_tensor(n, layers, params, run, hf_reference)
    return _mirror_upper(-2.0 * Q.imag, True).cpu().numpy()


def natural_gradient_direction(g: np.ndarray, gradient, regularization: float) -> np.ndarray:
    """(g + regularization I)^-1 gradient (vqe_natural_gradient_direction):
    a P x P solve with partial pivoting; a singular system raises."""
    A = np.array(g, dtype=np.float64, copy=True)
    A[np.diag_indices_from(A)] += regularization
    return np.linalg.solve(A, np.asarray(gradient, dtype=np.float64))
