"""Batched adjoint VQE gradients on the B200 engine, with a
`torch.autograd.Function` for the hardware-efficient ansatz energy.

The ansatz and gradient follow the reference's adjoint path
(vqe_build_hea_diff_circuit, vqe.c:1946-1981; moonlab_diff_backward_pauli_sum,
differentiable.c:478): X on the set bits of hf_reference, then per layer
RY/RZ on every qubit and a CNOT ladder; 2*N*L parameters.  The engine forms
lambda = H psi once and runs one backward sweep per batch (mlb_hea_*).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MlbError, check, load


def pauli_masks(paulis):
    """Pauli strings (char per qubit, index = qubit) -> (xmasks, zmasks)."""
    xs, zs = [], []
    for s in paulis:
        x = z = 0
        for q, ch in enumerate(s.upper()):
            if ch in "XY":
                x |= 1 << q
            if ch in "YZ":
                z |= 1 << q
            if ch not in "IXYZ":
                raise ValueError(f"invalid Pauli character {ch!r}")
        xs.append(x)
        zs.append(z)
    return np.array(xs, dtype=np.uint64), np.array(zs, dtype=np.uint64)


class HEAProblem:
    """E(theta) = <psi(theta)|H|psi(theta)> for the hardware-efficient ansatz."""

    def __init__(self, num_qubits: int, num_layers: int, coeffs, paulis=None, xmasks=None, zmasks=None,
                 hf_reference: int = 0, dtype: str = "c128", device: int = 0):
        self._lib = load()
        if paulis is not None:
            xmasks, zmasks = pauli_masks(paulis)
        x = np.ascontiguousarray(xmasks, dtype=np.uint64)
        z = np.ascontiguousarray(zmasks, dtype=np.uint64)
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        h = C.c_void_p()
        rc = self._lib.mlb_hea_create(num_qubits, num_layers, hf_reference, len(c),
                                      x.ctypes.data_as(C.POINTER(C.c_uint64)),
                                      z.ctypes.data_as(C.POINTER(C.c_uint64)),
                                      c.ctypes.data_as(C.POINTER(C.c_double)),
                                      _lib.MLB_C128 if dtype == "c128" else _lib.MLB_C64, device, C.byref(h))
        if rc:
            raise MlbError(rc, "mlb_hea_create", self._lib.mlb_hea_last_error().decode())
        self._h = h
        self.num_qubits, self.num_layers, self.dtype = num_qubits, num_layers, dtype
        self.num_parameters = 2 * num_qubits * num_layers

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.mlb_hea_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_memory_budget(self, nbytes: int) -> None:
        self._lib.mlb_hea_set_memory_budget(self._h, int(nbytes))

    def set_checkpointing(self, mode: str = "auto") -> None:
        """'auto' (checkpoints every ceil(sqrt(L)) layers when they fit beside
        the whole batch), 'always' or 'never'."""
        code = {"auto": 0, "always": 1, "never": -1}[mode]
        check(self._lib.mlb_hea_set_checkpointing(self._h, code), "mlb_hea_set_checkpointing")

    def set_fused_forward(self, mode: str = "auto") -> None:
        """complex64, N >= 13: the forward sweep on the tensor cores ('auto':
        on when planned, 'on', 'off')."""
        code = {"auto": 0, "on": 1, "off": -1}[mode]
        check(self._lib.mlb_hea_set_fused_forward(self._h, code), "mlb_hea_set_fused_forward")

    def last_eval_stats(self) -> dict:
        seg, used, chunks, fused = C.c_uint32(), C.c_int(), C.c_size_t(), C.c_int()
        fp, fb = C.c_uint32(), C.c_uint32()
        check(self._lib.mlb_hea_last_eval_stats(self._h, C.byref(seg), C.byref(used), C.byref(chunks)),
              "mlb_hea_last_eval_stats")
        check(self._lib.mlb_hea_last_forward_fused(self._h, C.byref(fused), C.byref(fp), C.byref(fb)),
              "mlb_hea_last_forward_fused")
        return {"segment_layers": seg.value, "checkpoints": bool(used.value), "sub_batches": chunks.value,
                "fused_forward": bool(fused.value), "fused_forward_passes": fp.value,
                "fused_forward_blocks": fb.value}

    def plan_stats(self):
        f, l, b = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._lib.mlb_hea_plan_stats(self._h, C.byref(f), C.byref(l), C.byref(b))
        return {"forward_passes": f.value, "lambda_passes": l.value, "backward_passes": b.value}

    def evaluate(self, params, want_grad: bool = True):
        """params [B, P] (numpy) -> (energies [B], grads [B, P] or None)."""
        p = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        B = p.shape[0]
        if p.shape[1] != self.num_parameters:
            raise ValueError(f"expected {self.num_parameters} parameters per vector")
        E = np.empty(B, dtype=np.float64)
        G = np.empty((B, self.num_parameters), dtype=np.float64) if want_grad else None
        rc = self._lib.mlb_hea_evaluate(self._h, B, p.ctypes.data, E.ctypes.data,
                                        G.ctypes.data if want_grad else None, 0)
        if rc:
            raise MlbError(rc, "mlb_hea_evaluate", self._lib.mlb_hea_last_error().decode())
        return E, G

    def geometry(self, params):
        """(metric g = Re Q, curvature F = -2 Im Q), each P x P, of the
        quantum geometric tensor at one parameter vector (complex128
        problems): psi and the P derivative states as one device batch and
        an FP64 Gram kernel (mlb_hea_geometry)."""
        p = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
        if p.size != self.num_parameters:
            raise ValueError(f"expected {self.num_parameters} parameters")
        P = self.num_parameters
        g = np.empty((P, P), dtype=np.float64)
        f = np.empty((P, P), dtype=np.float64)
        rc = self._lib.mlb_hea_geometry(self._h, p.ctypes.data, g.ctypes.data, f.ctypes.data)
        if rc:
            raise MlbError(rc, "mlb_hea_geometry", self._lib.mlb_hea_last_error().decode())
        return g, f

    def evaluate_torch(self, params, want_grad: bool = True):
        """params: torch float64 tensor [B, P] on cuda -> (E, G) cuda tensors."""
        import torch
        p = params.detach().contiguous().to(torch.float64)
        B = p.shape[0]
        E = torch.empty(B, dtype=torch.float64, device=p.device)
        G = torch.empty((B, self.num_parameters), dtype=torch.float64, device=p.device) if want_grad else None
        on_dev = 1 if p.is_cuda else 0
        if p.is_cuda:
            torch.cuda.current_stream(p.device).synchronize()
        rc = self._lib.mlb_hea_evaluate(self._h, B, p.data_ptr(), E.data_ptr(),
                                        G.data_ptr() if want_grad else None, on_dev)
        if rc:
            raise MlbError(rc, "mlb_hea_evaluate", self._lib.mlb_hea_last_error().decode())
        return E, G


def _make_function():
    import torch

    class AdjointEnergy(torch.autograd.Function):
        """E = AdjointEnergy.apply(params [B, P], problem): forward returns the
        B energies; backward returns grad_E[:, None] * dE/dtheta from the
        batched adjoint sweep (computed in the forward, one launch set)."""

        @staticmethod
        def forward(ctx, params, problem):
            E, G = problem.evaluate_torch(params, want_grad=params.requires_grad)
            if G is not None:
                ctx.save_for_backward(G)
            return E.to(params.dtype)

        @staticmethod
        def backward(ctx, grad_e):
            (G,) = ctx.saved_tensors
            return (grad_e.to(G.dtype)[:, None] * G), None

    return AdjointEnergy


def __getattr__(name):
    if name == "AdjointEnergy":
        return _make_function()
    raise AttributeError(name)
