"""Python mirror of the engine's C ABI: a GPU state vector with the
reference's gate, measurement and reduction vocabulary.

Names follow the reference's C functions (gate_rx, measurement_sample,
measurement_expectation_z, ...).  Every call goes through
libmoonlab_b200.so; nothing here computes on the host.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MlbGate, MlbOp, check, load
from .circuits import GATE_DTYPE


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class StateVector:
    """A 2^n-amplitude state on one GPU (complex128 by default)."""

    def __init__(self, num_qubits: int, dtype: str = "c128", device: int = 0):
        self._lib = load()
        self.n = int(num_qubits)
        self.dtype = dtype
        code = _lib.MLB_C128 if dtype == "c128" else _lib.MLB_C64
        h = C.c_void_p()
        check(self._lib.mlb_state_create(self.n, code, device, C.byref(h)), "mlb_state_create")
        self._h = h

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.mlb_state_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def dim(self) -> int:
        return 1 << self.n

    def set_exec_mode(self, mode: str) -> None:
        code = {"tiled": _lib.MLB_EXEC_TILED, "eager": _lib.MLB_EXEC_EAGER,
                "fused": _lib.MLB_EXEC_FUSED}[mode]
        check(self._lib.mlb_state_set_exec_mode(self._h, code), "mlb_state_set_exec_mode")

    def reset(self) -> None:
        check(self._lib.mlb_state_reset(self._h), "mlb_state_reset")

    def flush(self) -> None:
        check(self._lib.mlb_flush(self._h), "mlb_flush")

    def synchronize(self) -> None:
        check(self._lib.mlb_synchronize(self._h), "mlb_synchronize")

    def stream(self) -> int:
        """cudaStream_t (as an int) that this state's kernels run on."""
        p = C.c_void_p()
        check(self._lib.mlb_state_stream(self._h, C.byref(p)), "mlb_state_stream")
        return int(p.value or 0)

    def device_ptr(self) -> int:
        p = C.c_void_p()
        check(self._lib.mlb_state_device_ptr(self._h, C.byref(p)), "mlb_state_device_ptr")
        return int(p.value)

    def amplitudes(self) -> np.ndarray:
        out = np.empty(self.dim, dtype=np.complex128 if self.dtype == "c128" else np.complex64)
        check(self._lib.mlb_state_copy_to_host(self._h, out.ctypes.data_as(C.c_void_p)),
              "mlb_state_copy_to_host")
        return out

    def set_amplitudes(self, amps: np.ndarray) -> None:
        a = np.ascontiguousarray(amps, dtype=np.complex128 if self.dtype == "c128" else np.complex64)
        if a.size != self.dim:
            raise ValueError("amplitude count does not match the state")
        check(self._lib.mlb_state_copy_from_host(self._h, a.ctypes.data_as(C.c_void_p)),
              "mlb_state_copy_from_host")

    def copy_from(self, other: "StateVector") -> None:
        check(self._lib.mlb_state_copy(self._h, other._h), "mlb_state_copy")

    def flush_stats(self) -> dict:
        st = _lib.MlbFlushStats()
        check(self._lib.mlb_last_flush_stats(self._h, C.byref(st)), "mlb_last_flush_stats")
        return {f: getattr(st, f) for f, _ in st._fields_}

    def set_plan_cache(self, entries: int) -> None:
        check(self._lib.mlb_state_set_plan_cache(self._h, entries), "mlb_state_set_plan_cache")

    def set_dense(self, on: bool = True) -> None:
        """complex128 tiled mode: segments as dense matrices on the FP64
        tensor cores where they fit (default), or every segment gate by gate."""
        check(self._lib.mlb_state_set_dense(self._h, 1 if on else 0), "mlb_state_set_dense")

    def set_timing(self, enable: bool = True) -> None:
        check(self._lib.mlb_state_set_timing(self._h, 1 if enable else 0), "mlb_state_set_timing")

    # -- gates ---------------------------------------------------------------
    def apply_1q(self, target: int, m: np.ndarray) -> None:
        mm = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(4).view(np.float64))
        check(self._lib.mlb_apply_1q(self._h, target, _dptr(mm)), "mlb_apply_1q")

    def apply_2q(self, q0: int, q1: int, m: np.ndarray) -> None:
        mm = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(16).view(np.float64))
        check(self._lib.mlb_apply_2q(self._h, q0, q1, _dptr(mm)), "mlb_apply_2q")

    def apply_controlled_1q(self, controls, target: int, m: np.ndarray) -> None:
        mask = sum(1 << c for c in controls)
        mm = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(4).view(np.float64))
        check(self._lib.mlb_apply_controlled_1q(self._h, mask, target, _dptr(mm)),
              "mlb_apply_controlled_1q")

    def mcx(self, controls, target: int) -> None:
        check(self._lib.mlb_apply_mcx(self._h, sum(1 << c for c in controls), target), "mlb_apply_mcx")

    def mcz(self, qubits) -> None:
        check(self._lib.mlb_apply_mcz(self._h, sum(1 << q for q in qubits)), "mlb_apply_mcz")

    def cswap(self, controls, q0: int, q1: int) -> None:
        check(self._lib.mlb_apply_swap(self._h, sum(1 << c for c in controls), q0, q1), "mlb_apply_swap")

    def zz(self, q0: int, q1: int, theta: float) -> None:
        check(self._lib.mlb_apply_zz(self._h, q0, q1, theta), "mlb_apply_zz")

    def run(self, gates: np.ndarray) -> None:
        g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
        check(self._lib.mlb_run_gates(self._h, g.ctypes.data_as(C.POINTER(MlbGate)), len(g)),
              "mlb_run_gates")

    # -- reductions ----------------------------------------------------------
    def norm_sq(self) -> float:
        v = C.c_double()
        check(self._lib.mlb_norm_sq(self._h, C.byref(v)), "mlb_norm_sq")
        return v.value

    def probability_one_all(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(self._lib.mlb_prob_one_all(self._h, _dptr(out)), "mlb_prob_one_all")
        return out

    def expectation_z_all(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(self._lib.mlb_expect_z_all(self._h, _dptr(out)), "mlb_expect_z_all")
        return out

    def correlation_zz(self, q1: int, q2: int) -> float:
        v = C.c_double()
        check(self._lib.mlb_correlation_zz(self._h, q1, q2, C.byref(v)), "mlb_correlation_zz")
        return v.value

    def expectation_pauli(self, xmask: int, zmask: int) -> float:
        v = C.c_double()
        check(self._lib.mlb_expect_pauli(self._h, xmask, zmask, C.byref(v)), "mlb_expect_pauli")
        return v.value

    def expectation_pauli_sum(self, xmasks, zmasks, coeffs) -> float:
        x = np.ascontiguousarray(xmasks, dtype=np.uint64)
        z = np.ascontiguousarray(zmasks, dtype=np.uint64)
        c = np.ascontiguousarray(coeffs, dtype=np.float64)
        v = C.c_double()
        check(self._lib.mlb_expect_pauli_sum(self._h, len(x), x.ctypes.data_as(C.POINTER(C.c_uint64)),
                                             z.ctypes.data_as(C.POINTER(C.c_uint64)), _dptr(c),
                                             C.byref(v)), "mlb_expect_pauli_sum")
        return v.value

    def probabilities(self, rule: int = 0) -> np.ndarray:
        out = np.empty(self.dim, dtype=np.float64)
        check(self._lib.mlb_probabilities(self._h, rule, out.ctypes.data_as(C.c_void_p), None),
              "mlb_probabilities")
        return out

    # -- sampling / collapse -------------------------------------------------
    def sample(self, uniforms, rule: int = _lib.MLB_SAMPLE_CDF_GE) -> np.ndarray:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        out = np.empty(len(u), dtype=np.uint64)
        check(self._lib.mlb_sample(self._h, rule, _dptr(u), len(u),
                                   out.ctypes.data_as(C.POINTER(C.c_uint64))), "mlb_sample")
        return out

    def measure_qubit(self, q: int, u: float) -> int:
        r = C.c_int()
        check(self._lib.mlb_measure_qubit(self._h, q, u, C.byref(r)), "mlb_measure_qubit")
        return r.value

    def quantum_measure(self, q: int, u: float):
        r = C.c_int()
        p = C.c_double()
        check(self._lib.mlb_quantum_measure(self._h, q, u, C.byref(r), C.byref(p)), "mlb_quantum_measure")
        return r.value, p.value

    def measure_all(self, u: float) -> int:
        r = C.c_uint64()
        check(self._lib.mlb_measure_all(self._h, u, C.byref(r)), "mlb_measure_all")
        return int(r.value)

    def normalize(self) -> float:
        v = C.c_double()
        check(self._lib.mlb_normalize(self._h, C.byref(v)), "mlb_normalize")
        return v.value


def gates_to_ops(gates: np.ndarray, n: int):
    """Translate gate records to engine ops (host libm matrices)."""
    lib = load()
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    cnt = C.c_size_t()
    check(lib.mlb_gates_to_ops(g.ctypes.data_as(C.POINTER(MlbGate)), len(g), n, None, C.byref(cnt)),
          "mlb_gates_to_ops")
    ops = (MlbOp * cnt.value)()
    check(lib.mlb_gates_to_ops(g.ctypes.data_as(C.POINTER(MlbGate)), len(g), n, ops, C.byref(cnt)),
          "mlb_gates_to_ops")
    return ops


def fused_plan(gates: np.ndarray, n: int) -> dict:
    """The fused complex64 path's plan for a circuit (host only): passes
    (tile high qubits, block range), blocks (tile bit positions, row bits,
    image index) and the bf16 operand images, as mlb_fused_plan returns them."""
    from ._lib import MlbFusedBlock, MlbFusedPass
    lib = load()
    ops = gates_to_ops(gates, n)
    np_, nb, ib = C.c_size_t(), C.c_size_t(), C.c_size_t()
    check(lib.mlb_fused_plan(ops, len(ops), n, None, C.byref(np_), None, C.byref(nb), None, C.byref(ib)),
          "mlb_fused_plan")
    passes = (MlbFusedPass * np_.value)()
    blocks = (MlbFusedBlock * nb.value)()
    images = np.empty(ib.value, dtype=np.uint8)
    check(lib.mlb_fused_plan(ops, len(ops), n, passes, C.byref(np_), blocks, C.byref(nb),
                             images.ctypes.data_as(C.c_void_p), C.byref(ib)), "mlb_fused_plan")
    return {
        "passes": [{"hbits": list(p.hbits)[:p.num_high], "num_low": p.num_low, "num_tiles": p.num_tiles,
                    "block_begin": p.block_begin, "num_blocks": p.num_blocks} for p in passes],
        "blocks": [{"pos": list(b.pos), "rows": list(b.rows), "image": b.image} for b in blocks],
        "images": images,
    }
