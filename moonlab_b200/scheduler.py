"""Scheduler jobs on the engine (reference src/distributed/scheduler.{h,c}).

`parse_job_json` reads the text of the reference's moonlab_job_to_json;
`parse_circuit_text` / `format_circuit_text` read and write the
"moonlab-circuit v1" text of moonlab_qgtl_circuit_serialize
(src/applications/moonlab_qgtl_backend.c:319-506);
`run_job` executes a job with the default "simulator" backend's semantics
(worker slices, splitmix64 worker seeds, xorshift64 uniforms, one
measurement_all_qubits per shot) on the GPU; `register_backend` adds the
"b200" backend to the scheduler registry of a loaded reference library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .circuits import GATE_DTYPE
from ._lib import check


def parse_job_json(text: str):
    """(desc dict, gate records of GATE_DTYPE) from moonlab_job_to_json text."""
    lib = _lib.load()
    raw = text.encode()
    d = _lib.MlbJobDesc()
    n = C.c_size_t()
    check(lib.mlb_job_parse_json(raw, C.byref(d), None, 0, C.byref(n)), "mlb_job_parse_json")
    gates = np.zeros(n.value, dtype=GATE_DTYPE)
    check(lib.mlb_job_parse_json(raw, C.byref(d), gates.ctypes.data_as(C.c_void_p), n.value, C.byref(n)),
          "mlb_job_parse_json")
    desc = {"num_qubits": d.num_qubits, "num_shots": d.num_shots, "num_workers": d.num_workers,
            "rng_seed": int(d.rng_seed)}
    return desc, gates


def parse_circuit_text(text):
    """(num_qubits, gate records of GATE_DTYPE) from "moonlab-circuit v1"
    text (str or bytes; its whole length is read, so a NUL inside is
    invalid input, as for the reference's deserializer given a length)."""
    lib = _lib.load()
    raw = text.encode() if isinstance(text, str) else bytes(text)
    if not raw:
        raise ValueError("empty circuit text")
    nq = C.c_uint32()
    n = C.c_size_t()
    check(lib.mlb_circuit_parse_text(raw, len(raw), C.byref(nq), None, 0, C.byref(n)), "mlb_circuit_parse_text")
    gates = np.zeros(n.value, dtype=GATE_DTYPE)
    check(lib.mlb_circuit_parse_text(raw, len(raw), C.byref(nq), gates.ctypes.data_as(C.c_void_p), n.value,
                                     C.byref(n)), "mlb_circuit_parse_text")
    return int(nq.value), gates


def format_circuit_text(num_qubits: int, gates: np.ndarray) -> str:
    """The reference serializer's text for gate records of types 0..13."""
    lib = _lib.load()
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    w = C.c_size_t()
    check(lib.mlb_circuit_format_text(num_qubits, g.ctypes.data_as(C.c_void_p), len(g), None, 0, C.byref(w)),
          "mlb_circuit_format_text")
    buf = C.create_string_buffer(w.value + 1)
    check(lib.mlb_circuit_format_text(num_qubits, g.ctypes.data_as(C.c_void_p), len(g), buf, len(buf),
                                      C.byref(w)), "mlb_circuit_format_text")
    return buf.value.decode()


def run_job(num_qubits: int, gates: np.ndarray, num_shots: int, num_workers: int = 1,
            rng_seed: int = 0, device: int = 0):
    """outcomes[num_shots] (uint64), workers used, wall seconds."""
    lib = _lib.load()
    g = np.ascontiguousarray(gates, dtype=GATE_DTYPE)
    d = _lib.MlbJobDesc(num_qubits, num_shots, num_workers, 0, rng_seed)
    out = np.empty(num_shots, dtype=np.uint64)
    w = C.c_int()
    secs = C.c_double()
    check(lib.mlb_job_run(C.byref(d), g.ctypes.data_as(C.c_void_p), len(g), device,
                          out.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(w), C.byref(secs)),
          "mlb_job_run")
    return out, w.value, secs.value


def register_backend(reference_lib=None) -> int:
    """Register "b200" with the reference scheduler.  reference_lib: a ctypes
    handle of libquantumsim (needed when it was opened RTLD_LOCAL); without
    it the registry is looked up in the global symbol scope.  Returns the
    registry's status code (0 = MOONLAB_SCHED_OK)."""
    lib = _lib.load()
    if reference_lib is None:
        return lib.moonlab_b200_register_backend()
    reg = C.cast(reference_lib.moonlab_register_backend, C.c_void_p)
    to_json = C.cast(reference_lib.moonlab_job_to_json, C.c_void_p)
    return lib.moonlab_b200_register_backend_with(reg, to_json)
