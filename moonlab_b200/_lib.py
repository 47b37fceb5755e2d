"""ctypes binding of libmoonlab_b200.so (include/moonlab_b200.h).

The library is loaded RTLD_GLOBAL so that its strong definitions of the
reference's GPU-routing symbols (quantum_state_create_gpu, qsim_gpu_route_*,
moonlab_cuda_*) are visible to a reference core library loaded afterwards.
There is no fallback: if the library is missing, importing this module
raises, naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libmoonlab_b200.so"

MLB_OK = 0
STATUS_NAMES = {
    0: "MLB_OK", -1: "MLB_ERR_OUT_OF_MEMORY", -2: "MLB_ERR_NO_DEVICE", -3: "MLB_ERR_DRIVER",
    -4: "MLB_ERR_INVALID_QUBIT", -5: "MLB_ERR_NUM_QUBITS", -6: "MLB_ERR_INVALID_ARG",
    -7: "MLB_ERR_TIMEOUT", -8: "MLB_ERR_BUSY", -9: "MLB_ERR_NOT_SUPPORTED",
}
MLB_C128, MLB_C64 = 0, 1
MLB_EXEC_TILED, MLB_EXEC_EAGER, MLB_EXEC_FUSED = 0, 1, 2
MLB_OP_1Q, MLB_OP_2Q, MLB_OP_DIAG1, MLB_OP_X, MLB_OP_SWAP, MLB_OP_ZZ, MLB_OP_PHASE = range(7)
MLB_SAMPLE_CDF_GE, MLB_SAMPLE_CUM_GT = 0, 1


class MlbOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("target", C.c_int32), ("target2", C.c_int32),
                ("reserved", C.c_int32), ("cmask", C.c_uint64), ("m", C.c_double * 32)]


class MlbGate(C.Structure):
    _fields_ = [("type", C.c_int32), ("target", C.c_int32), ("control", C.c_int32),
                ("reserved", C.c_int32), ("theta", C.c_double)]


class MlbFlushStats(C.Structure):
    _fields_ = [("passes", C.c_uint64), ("ops", C.c_uint64), ("dense_blocks", C.c_uint64),
                ("bytes_moved", C.c_uint64), ("kernel_launches", C.c_uint64), ("segments", C.c_uint64),
                ("gpu_ms", C.c_double), ("plan_cache_hit", C.c_uint64), ("dense_amps", C.c_uint64)]


class MlbJobDesc(C.Structure):
    _fields_ = [("num_qubits", C.c_int32), ("num_shots", C.c_int32), ("num_workers", C.c_int32),
                ("reserved", C.c_int32), ("rng_seed", C.c_uint64)]


class MlbFusedPass(C.Structure):
    _fields_ = [("hbits", C.c_uint8 * 12), ("num_low", C.c_uint8), ("num_high", C.c_uint8),
                ("reserved", C.c_uint8 * 2), ("num_tiles", C.c_uint64), ("block_begin", C.c_uint32),
                ("num_blocks", C.c_uint32)]


class MlbTilePass(C.Structure):
    _fields_ = [("high", C.c_uint8 * 16), ("num_low", C.c_uint8), ("num_high", C.c_uint8),
                ("reserved", C.c_uint8 * 2), ("seg_begin", C.c_uint32), ("num_segments", C.c_uint32)]


class MlbTileSegment(C.Structure):
    _fields_ = [("mode", C.c_int32), ("nbits", C.c_int32), ("bits", C.c_int32 * 4), ("op_begin", C.c_uint32),
                ("op_end", C.c_uint32)]


class MlbFusedBlock(C.Structure):
    _fields_ = [("pos", C.c_uint8 * 5), ("rows", C.c_uint8 * 8), ("reserved", C.c_uint8 * 3),
                ("image", C.c_uint32)]


class QuantumState(C.Structure):
    """quantum_state_t (reference src/quantum/state.h:102-131)."""
    _fields_ = [("num_qubits", C.c_size_t), ("state_dim", C.c_size_t), ("amplitudes", C.c_void_p),
                ("measurement_outcomes", C.c_void_p), ("num_measurements", C.c_size_t),
                ("max_measurements", C.c_size_t), ("owns_memory", C.c_int),
                ("gpu_state", C.c_void_p), ("gpu_backend", C.c_int)]


class MlbError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{what}: {name}" + (f" ({detail})" if detail else ""))


_SIGS = {
    # name: (restype, argtypes)
    "mlb_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "mlb_state_create": (C.c_int, [C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mlb_state_free": (None, [C.c_void_p]),
    "mlb_state_num_qubits": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "mlb_state_dim": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "mlb_state_dtype": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "mlb_state_device_ptr": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mlb_state_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mlb_state_set_exec_mode": (C.c_int, [C.c_void_p, C.c_int]),
    "mlb_state_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mlb_state_reset": (C.c_int, [C.c_void_p]),
    "mlb_state_copy_to_host": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mlb_state_copy_from_host": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mlb_state_copy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mlb_flush": (C.c_int, [C.c_void_p]),
    "mlb_synchronize": (C.c_int, [C.c_void_p]),
    "mlb_apply_op": (C.c_int, [C.c_void_p, C.POINTER(MlbOp)]),
    "mlb_apply_ops": (C.c_int, [C.c_void_p, C.POINTER(MlbOp), C.c_size_t]),
    "mlb_apply_1q": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "mlb_apply_2q": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]),
    "mlb_apply_controlled_1q": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.POINTER(C.c_double)]),
    "mlb_apply_mcx": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32]),
    "mlb_apply_mcz": (C.c_int, [C.c_void_p, C.c_uint64]),
    "mlb_apply_swap": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32]),
    "mlb_apply_zz": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_double]),
    "mlb_norm_sq": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mlb_prob_one": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "mlb_prob_one_all": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mlb_prob_one_all_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p]),
    "mlb_expect_z_all": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mlb_prob_one_exact": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "mlb_correlation_zz": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]),
    "mlb_expect_pauli": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.POINTER(C.c_double)]),
    "mlb_expect_pauli_sum": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_uint64), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]),
    "mlb_probabilities": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "mlb_sample": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_size_t,
                             C.POINTER(C.c_uint64)]),
    "mlb_measure_qubit": (C.c_int, [C.c_void_p, C.c_uint32, C.c_double, C.POINTER(C.c_int)]),
    "mlb_quantum_measure": (C.c_int, [C.c_void_p, C.c_uint32, C.c_double, C.POINTER(C.c_int),
                                      C.POINTER(C.c_double)]),
    "mlb_measure_all": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_uint64)]),
    "mlb_normalize": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mlb_gates_to_ops": (C.c_int, [C.POINTER(MlbGate), C.c_size_t, C.c_uint32, C.POINTER(MlbOp),
                                   C.POINTER(C.c_size_t)]),
    "mlb_run_gates": (C.c_int, [C.c_void_p, C.POINTER(MlbGate), C.c_size_t]),
    "mlb_last_flush_stats": (C.c_int, [C.c_void_p, C.POINTER(MlbFlushStats)]),
    "mlb_state_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "mlb_test_fused_skip_copy": (C.c_int, [C.c_void_p]),
    "mlb_state_set_plan_cache": (C.c_int, [C.c_void_p, C.c_size_t]),
    "mlb_state_set_dense": (C.c_int, [C.c_void_p, C.c_int]),
    "mlb_plan_ops": (C.c_int, [C.POINTER(MlbOp), C.c_size_t, C.c_uint32, C.c_int, C.c_int,
                               C.POINTER(MlbFlushStats)]),
    "mlb_total_kernel_launches": (C.c_int, [C.POINTER(C.c_uint64)]),
    "mlb_tile_plan": (C.c_int, [C.POINTER(MlbOp), C.c_size_t, C.c_uint32, C.c_int, C.c_int,
                                C.POINTER(MlbTilePass), C.POINTER(C.c_size_t), C.POINTER(MlbTileSegment),
                                C.POINTER(C.c_size_t), C.POINTER(MlbOp), C.POINTER(C.c_size_t)]),
    "mlb_fused_plan": (C.c_int, [C.POINTER(MlbOp), C.c_size_t, C.c_uint32, C.POINTER(MlbFusedPass),
                                 C.POINTER(C.c_size_t), C.POINTER(MlbFusedBlock), C.POINTER(C.c_size_t),
                                 C.c_void_p, C.POINTER(C.c_size_t)]),
    "mlb_hea_create": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint64, C.c_size_t, C.POINTER(C.c_uint64),
                                 C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.c_int, C.c_int,
                                 C.POINTER(C.c_void_p)]),
    "mlb_hea_free": (None, [C.c_void_p]),
    "mlb_hea_num_parameters": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "mlb_hea_evaluate": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "mlb_hea_set_memory_budget": (C.c_int, [C.c_void_p, C.c_size_t]),
    "mlb_hea_plan_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint32)]),
    "mlb_hea_last_error": (C.c_char_p, []),
    "mlb_hea_set_checkpointing": (C.c_int, [C.c_void_p, C.c_int]),
    "mlb_hea_set_fused_forward": (C.c_int, [C.c_void_p, C.c_int]),
    "mlb_hea_last_forward_fused": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_uint32),
                                             C.POINTER(C.c_uint32)]),
    "mlb_hea_last_eval_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_int),
                                          C.POINTER(C.c_size_t)]),
    "moonlab_vqe_gradient": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_size_t]),
    "mlb_hea_geometry": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "moonlab_vqe_qgt": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_size_t]),
    "moonlab_vqe_berry_curvature": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                              C.c_size_t]),
    "moonlab_vqe_natural_gradient": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                               C.c_double, C.POINTER(C.c_double), C.c_size_t]),
    "moonlab_b200_vqe_gradient_batch": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_double),
                                                  C.POINTER(C.c_double), C.c_size_t]),
    "mlb_job_parse_json": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                     C.POINTER(C.c_size_t)]),
    "mlb_circuit_parse_text": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_uint32), C.c_void_p,
                                         C.c_size_t, C.POINTER(C.c_size_t)]),
    "mlb_circuit_format_text": (C.c_int, [C.c_uint32, C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t,
                                          C.POINTER(C.c_size_t)]),
    "mlb_fp64_tensor_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "mlb_control_create": (C.c_int, [C.c_int, C.c_size_t, C.c_int, C.c_uint32, C.POINTER(C.c_void_p)]),
    "mlb_control_set_seed": (C.c_int, [C.c_void_p, C.c_uint64]),
    "mlb_control_handle": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_size_t)]),
    "mlb_control_free": (None, [C.c_void_p]),
    "mlb_control_destroy": (None, [C.c_void_p]),
    "mlb_job_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.POINTER(C.c_uint64),
                              C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "moonlab_b200_backend_execute": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "moonlab_b200_register_backend": (C.c_int, []),
    "moonlab_b200_register_backend_with": (C.c_int, [C.c_void_p, C.c_void_p]),
    "moonlab_b200_release_backend_state": (None, []),
    "mlb_status_string": (C.c_char_p, [C.c_int]),
    "mlb_last_error": (C.c_char_p, []),
    # reference-compatible drop-in surface
    "quantum_state_create_gpu": (C.c_int, [C.c_size_t, C.POINTER(C.POINTER(QuantumState))]),
    "quantum_state_sync_to_host": (C.c_int, [C.POINTER(QuantumState)]),
    "quantum_state_sync_from_host": (C.c_int, [C.POINTER(QuantumState)]),
    "qsim_gpu_route_hadamard": (C.c_int, [C.POINTER(QuantumState), C.c_int]),
    "qsim_gpu_route_pauli_x": (C.c_int, [C.POINTER(QuantumState), C.c_int]),
    "qsim_gpu_route_cnot": (C.c_int, [C.POINTER(QuantumState), C.c_int, C.c_int]),
    "qsim_gpu_route_apply_1q_matrix": (C.c_int, [C.POINTER(QuantumState), C.c_int, C.POINTER(C.c_double)]),
    "qsim_gpu_route_apply_2q_matrix": (C.c_int, [C.POINTER(QuantumState), C.c_int, C.c_int,
                                                 C.POINTER(C.c_double)]),
    "qsim_gpu_route_mcx": (C.c_int, [C.POINTER(QuantumState), C.c_uint64, C.c_int]),
    "qsim_gpu_route_mcz": (C.c_int, [C.POINTER(QuantumState), C.c_uint64]),
    "qsim_gpu_route_fredkin": (C.c_int, [C.POINTER(QuantumState), C.c_int, C.c_int, C.c_int]),
    "moonlab_cuda_state_create": (C.c_int, [C.c_uint32, C.POINTER(C.c_void_p)]),
    "moonlab_cuda_state_free": (None, [C.c_void_p]),
    "moonlab_cuda_state_n_qubits": (C.c_uint32, [C.c_void_p]),
    "moonlab_cuda_state_dim": (C.c_uint64, [C.c_void_p]),
    "moonlab_cuda_apply_1q": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "moonlab_cuda_apply_cnot": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "moonlab_cuda_apply_2q": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_double)]),
    "moonlab_cuda_prob_z": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "moonlab_cuda_norm": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "moonlab_cuda_apply_x": (C.c_int, [C.c_void_p, C.c_uint32]),
    "moonlab_cuda_apply_h": (C.c_int, [C.c_void_p, C.c_uint32]),
    "moonlab_cuda_state_copy_to_host": (C.c_int, [C.c_void_p, C.c_void_p]),
    "moonlab_cuda_state_copy_from_host": (C.c_int, [C.c_void_p, C.c_void_p]),
    "moonlab_cuda_apply_mcx": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint32]),
    "moonlab_cuda_apply_mcz": (C.c_int, [C.c_void_p, C.c_uint64]),
    "moonlab_cuda_apply_fredkin": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32]),
    "moonlab_cuda_synchronize": (C.c_int, [C.c_void_p]),
    "moonlab_cuda_runtime_probe_discrete": (C.c_int, []),
    "moonlab_cuda_select_device_for_rank": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "moonlab_b200_engine_of": (C.c_void_p, [C.POINTER(QuantumState)]),
}

_lib = None


def load() -> C.CDLL:
    """Load libmoonlab_b200.so (built by __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(or `make -C moonlab_b200/csrc`). The engine has no CPU fallback.")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue  # exported_symbols() reports what is missing
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> dict:
    lib = load()
    return {name: hasattr(lib, name) for name in _SIGS}


def check(status: int, what: str) -> None:
    if status != MLB_OK:
        detail = load().mlb_last_error()
        raise MlbError(status, what, detail.decode() if detail else "")


def kernel_launches() -> int:
    v = C.c_uint64()
    check(load().mlb_total_kernel_launches(C.byref(v)), "mlb_total_kernel_launches")
    return int(v.value)
