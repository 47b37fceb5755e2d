"""ctypes bindings of the two CPU oracles.  TEST INFRASTRUCTURE ONLY: used
by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by
the engine.

* Port  -- oracle/libsv_oracle.so, the plain-C restatement (sv_oracle.c).
* Ref   -- oracle/_ref/liboracle.so, the reference's own CPU implementation
           compiled from its sources by oracle/Makefile (present only where
           the reference tree was available at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
PORT_LIB = ORACLE_DIR / "libsv_oracle.so"
REF_LIB = ORACLE_DIR / "_ref" / "liboracle.so"
REF_DROPIN_LIB = ORACLE_DIR / "_ref" / "libref_dropin.so"

SVO = dict(I=0, X=1, Y=2, Z=3, H=4, S=5, T=6, RX=7, RY=8, RZ=9, CNOT=10, CY=11, CZ=12, SWAP=13,
           SDG=20, TDG=21, PHASE=22, CPHASE=23, CRX=24, CRY=25, CRZ=26, ZZ=27, TOFFOLI=28,
           FREDKIN=29, U3=30)


class SvoGate(C.Structure):
    _fields_ = [("type", C.c_int32), ("q0", C.c_int32), ("q1", C.c_int32), ("q2", C.c_int32),
                ("theta", C.c_double), ("theta2", C.c_double), ("theta3", C.c_double)]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _u64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


# ---------------------------------------------------------------------------
# the C restatement
# ---------------------------------------------------------------------------
_port = None


def port():
    global _port
    if _port is None:
        if not PORT_LIB.exists():
            subprocess.run(["make", "-C", str(ORACLE_DIR), "port"], check=True,
                           stdout=subprocess.DEVNULL)
        lib = C.CDLL(str(PORT_LIB))
        dp, u64p, i, u64, d, sz = (C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.c_int,
                                   C.c_uint64, C.c_double, C.c_size_t)
        sigs = {
            "svo_init_zero": (None, [dp, i]),
            "svo_apply_gate": (i, [dp, i, C.POINTER(SvoGate)]),
            "svo_apply_circuit": (i, [dp, i, C.POINTER(SvoGate), sz]),
            "svo_apply_1q_matrix": (None, [dp, i, i, dp]),
            "svo_apply_2q_matrix": (None, [dp, i, i, i, dp]),
            "svo_apply_mcx": (None, [dp, i, u64, i]),
            "svo_apply_mcz": (None, [dp, i, u64]),
            "svo_probability_one": (d, [dp, i, i]),
            "svo_probability_distribution": (None, [dp, i, dp]),
            "svo_qgtl_probabilities": (None, [dp, i, dp]),
            "svo_expectation_z": (d, [dp, i, i]),
            "svo_expectation_x": (d, [dp, i, i]),
            "svo_expectation_y": (d, [dp, i, i]),
            "svo_correlation_zz": (d, [dp, i, i, i]),
            "svo_norm_sq": (d, [dp, i]),
            "svo_expect_pauli_string": (d, [dp, i, u64, u64]),
            "svo_measurement_sample": (None, [dp, i, u64p, i, dp]),
            "svo_measure_all_index": (u64, [dp, i, d]),
            "svo_measurement_single_qubit": (i, [dp, i, i, d]),
            "svo_quantum_measure": (i, [dp, i, i, d, dp]),
            "svo_qgtl_execute": (i, [i, C.POINTER(SvoGate), sz, i, u64, u64p, dp]),
            "svo_scheduler_simulator": (i, [i, C.POINTER(SvoGate), sz, i, i, u64, u64p]),
            "svo_hea_energy_and_gradient": (i, [i, i, u64, dp, sz, dp, C.c_char_p, dp, dp]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _port = lib
    return _port


def to_svo(gates) -> "C.Array":
    """QGTL-numbered gate records (moonlab_b200.circuits.GATE_DTYPE) to svo_gate_t.
    Two-qubit records: control -> q0, target -> q1 (SWAP: qubit1, qubit2)."""
    arr = (SvoGate * len(gates))()
    for k, g in enumerate(gates):
        t, tgt, ctl, th = int(g["type"]), int(g["target"]), int(g["control"]), float(g["theta"])
        if t in (10, 11, 12, 13, 23, 24, 25, 26, 27):
            arr[k] = SvoGate(t, ctl, tgt, -1, th, 0.0, 0.0)
        else:
            arr[k] = SvoGate(t, tgt, -1, -1, th, 0.0, 0.0)
    return arr


def port_run(n: int, gates) -> np.ndarray:
    lib = port()
    a = np.zeros(1 << n, dtype=np.complex128)
    av = a.view(np.float64)
    lib.svo_init_zero(_dp(av), n)
    g = to_svo(gates)
    rc = lib.svo_apply_circuit(_dp(av), n, g, len(g))
    if rc:
        raise RuntimeError(f"svo_apply_circuit failed: {rc}")
    return a


def port_run_from(n: int, gates, state) -> np.ndarray:
    """Gate records applied to a given state (copy) by the restatement."""
    a = np.array(state, dtype=np.complex128, copy=True)
    g = to_svo(gates)
    rc = port().svo_apply_circuit(_dp(a.view(np.float64)), n, g, len(g))
    if rc:
        raise RuntimeError(f"svo_apply_circuit failed: {rc}")
    return a


def port_probabilities(a: np.ndarray, rule: int = 0) -> np.ndarray:
    lib = port()
    n = int(a.size).bit_length() - 1
    out = np.empty(a.size, dtype=np.float64)
    av = np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)
    (lib.svo_probability_distribution if rule == 0 else lib.svo_qgtl_probabilities)(_dp(av), n, _dp(out))
    return out


def port_sample(a: np.ndarray, uniforms) -> np.ndarray:
    lib = port()
    n = int(a.size).bit_length() - 1
    u = np.ascontiguousarray(uniforms, dtype=np.float64)
    out = np.empty(len(u), dtype=np.uint64)
    av = np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)
    lib.svo_measurement_sample(_dp(av), n, _u64p(out), len(u), _dp(u))
    return out


def port_measure_all_indices(a: np.ndarray, uniforms) -> np.ndarray:
    lib = port()
    n = int(a.size).bit_length() - 1
    av = np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)
    return np.array([lib.svo_measure_all_index(_dp(av), n, float(u)) for u in uniforms], dtype=np.uint64)


# ---------------------------------------------------------------------------
# the reference's own library
# ---------------------------------------------------------------------------
class RefState(C.Structure):
    """quantum_state_t (src/quantum/state.h:102-131)."""
    _fields_ = [("num_qubits", C.c_size_t), ("state_dim", C.c_size_t), ("amplitudes", C.c_void_p),
                ("measurement_outcomes", C.c_void_p), ("num_measurements", C.c_size_t),
                ("max_measurements", C.c_size_t), ("owns_memory", C.c_int),
                ("gpu_state", C.c_void_p), ("gpu_backend", C.c_int)]


class QgtlOpts(C.Structure):
    _fields_ = [("num_shots", C.c_int), ("rng_seed", C.c_uint64), ("return_probabilities", C.c_int)]


class QgtlResults(C.Structure):
    _fields_ = [("num_qubits", C.c_int), ("num_shots", C.c_int), ("outcomes", C.POINTER(C.c_uint64)),
                ("probabilities", C.POINTER(C.c_double))]


class JobResults(C.Structure):
    _fields_ = [("num_qubits", C.c_int), ("total_shots", C.c_int), ("outcomes", C.POINTER(C.c_uint64)),
                ("num_workers_used", C.c_int), ("worker_seconds", C.POINTER(C.c_double))]


ENTROPY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint8), C.c_size_t)


class EntropyCtx(C.Structure):
    _fields_ = [("get_bytes", ENTROPY_FN), ("user_data", C.c_void_p)]


_ref = None


def have_ref() -> bool:
    return REF_LIB.exists()


def ref():
    """The reference's library (liboracle.so) with the signatures tests use."""
    global _ref
    if _ref is None:
        # RTLD_DEEPBIND: the reference resolves its own symbols first, so the
        # drop-in's definitions of the same names (loaded globally, e.g.
        # fuse_circuit_create) never stand in for the reference's internals
        lib = C.CDLL(str(REF_LIB), mode=os.RTLD_LOCAL | os.RTLD_DEEPBIND)
        sp = C.POINTER(RefState)
        i, d, u64, sz = C.c_int, C.c_double, C.c_uint64, C.c_size_t
        sigs = {
            "quantum_state_init": (i, [sp, sz]), "quantum_state_free": (None, [sp]),
            "gate_pauli_x": (i, [sp, i]), "gate_pauli_y": (i, [sp, i]), "gate_pauli_z": (i, [sp, i]),
            "gate_hadamard": (i, [sp, i]), "gate_s": (i, [sp, i]), "gate_s_dagger": (i, [sp, i]),
            "gate_t": (i, [sp, i]), "gate_t_dagger": (i, [sp, i]), "gate_phase": (i, [sp, i, d]),
            "gate_rx": (i, [sp, i, d]), "gate_ry": (i, [sp, i, d]), "gate_rz": (i, [sp, i, d]),
            "gate_u3": (i, [sp, i, d, d, d]),
            "gate_cnot": (i, [sp, i, i]), "gate_cz": (i, [sp, i, i]), "gate_cy": (i, [sp, i, i]),
            "gate_swap": (i, [sp, i, i]), "gate_cphase": (i, [sp, i, i, d]),
            "gate_crx": (i, [sp, i, i, d]), "gate_cry": (i, [sp, i, i, d]), "gate_crz": (i, [sp, i, i, d]),
            "gate_toffoli": (i, [sp, i, i, i]), "gate_fredkin": (i, [sp, i, i, i]),
            "measurement_probability_one": (d, [sp, i]),
            "measurement_probability_distribution": (None, [sp, C.POINTER(d)]),
            "measurement_expectation_z": (d, [sp, i]), "measurement_expectation_x": (d, [sp, i]),
            "measurement_expectation_y": (d, [sp, i]), "measurement_correlation_zz": (d, [sp, i, i]),
            "measurement_sample": (None, [sp, C.POINTER(u64), i, C.POINTER(d)]),
            "measurement_all_qubits": (u64, [sp, d]),
            "measurement_single_qubit": (i, [sp, i, d]),
            "quantum_state_clone": (i, [sp, sp]),
            "moonlab_qgtl_circuit_create": (C.c_void_p, [i]),
            "moonlab_qgtl_circuit_free": (None, [C.c_void_p]),
            "moonlab_qgtl_add_gate": (i, [C.c_void_p, i, i, i, C.POINTER(d)]),
            "moonlab_qgtl_execute": (i, [C.c_void_p, C.POINTER(QgtlOpts), C.POINTER(QgtlResults)]),
            "moonlab_qgtl_results_free": (None, [C.POINTER(QgtlResults)]),
            "moonlab_qgtl_circuit_num_gates": (i, [C.c_void_p]),
            "moonlab_qgtl_circuit_serialize": (i, [C.c_void_p, C.c_char_p, sz, C.POINTER(sz)]),
            "moonlab_qgtl_circuit_deserialize": (C.c_void_p, [C.c_char_p, sz, C.POINTER(i)]),
            "moonlab_job_create": (C.c_void_p, [i]), "moonlab_job_free": (None, [C.c_void_p]),
            "moonlab_job_add_gate": (i, [C.c_void_p, i, i, i, C.POINTER(d)]),
            "moonlab_job_set_num_shots": (i, [C.c_void_p, i]),
            "moonlab_job_set_num_workers": (i, [C.c_void_p, i]),
            "moonlab_job_set_rng_seed": (i, [C.c_void_p, u64]),
            "moonlab_job_to_json": (i, [C.c_void_p, C.c_char_p, sz]),
            "moonlab_scheduler_run": (i, [C.c_void_p, C.POINTER(JobResults)]),
            "moonlab_job_results_free": (None, [C.POINTER(JobResults)]),
            "fuse_circuit_create": (C.c_void_p, [sz]), "fuse_circuit_free": (None, [C.c_void_p]),
            "fuse_circuit_len": (sz, [C.c_void_p]), "fuse_compile": (C.c_void_p, [C.c_void_p, C.c_void_p]),
            "fuse_execute": (i, [C.c_void_p, sp]),
            "fuse_append_u3": (i, [C.c_void_p, i, d, d, d]),
            "pauli_hamiltonian_create": (C.c_void_p, [sz, sz]),
            "pauli_hamiltonian_add_term": (i, [C.c_void_p, d, C.c_char_p, sz]),
            "vqe_create_hardware_efficient_ansatz": (C.c_void_p, [sz, sz]),
            "vqe_create_uccsd_ansatz": (C.c_void_p, [sz, sz]),
            "vqe_create_symmetry_preserving_ansatz": (C.c_void_p, [sz, sz, sz]),
            "vqe_compute_gradient": (i, [C.c_void_p, C.POINTER(d), C.POINTER(d)]),
            "moonlab_vqe_natural_gradient": (i, [C.c_void_p, C.POINTER(d), C.POINTER(d), d, C.POINTER(d), sz]),
            "vqe_optimizer_create": (C.c_void_p, [i]),
            "vqe_solver_create": (C.c_void_p, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
            "vqe_solver_free": (None, [C.c_void_p]),
            "moonlab_vqe_gradient": (i, [C.c_void_p, C.POINTER(d), C.POINTER(d), sz]),
            "moonlab_vqe_qgt": (i, [C.c_void_p, C.POINTER(d), C.POINTER(d), sz]),
            "moonlab_vqe_berry_curvature": (i, [C.c_void_p, C.POINTER(d), C.POINTER(d), sz]),
            "vqe_natural_gradient_direction": (i, [C.c_void_p, C.POINTER(d), C.POINTER(d), d, C.POINTER(d)]),
        }
        for k in ("h", "x", "y", "z", "s", "sdg", "t", "tdg"):
            sigs[f"fuse_append_{k}"] = (i, [C.c_void_p, i])
        for k in ("phase", "rx", "ry", "rz"):
            sigs[f"fuse_append_{k}"] = (i, [C.c_void_p, i, d])
        for k in ("cnot", "cz", "cy", "swap"):
            sigs[f"fuse_append_{k}"] = (i, [C.c_void_p, i, i])
        for k in ("cphase", "crx", "cry", "crz"):
            sigs[f"fuse_append_{k}"] = (i, [C.c_void_p, i, i, d])
        for name, (res, args) in sigs.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _ref = lib
    return _ref


class RefStateVector:
    """A reference CPU state driven through the reference's gate_* API."""

    def __init__(self, n: int):
        self.lib = ref()
        self.s = RefState()
        rc = self.lib.quantum_state_init(C.byref(self.s), n)
        if rc:
            raise RuntimeError(f"quantum_state_init failed: {rc}")
        self.n = n

    def amplitudes(self) -> np.ndarray:
        buf = (C.c_double * (2 << self.n)).from_address(self.s.amplitudes)
        return np.frombuffer(buf, dtype=np.complex128).copy()

    def set_amplitudes(self, a: np.ndarray) -> None:
        buf = (C.c_double * (2 << self.n)).from_address(self.s.amplitudes)
        np.frombuffer(buf, dtype=np.complex128)[:] = a

    def run(self, gates) -> None:
        L, p = self.lib, C.byref(self.s)
        for g in gates:
            t, tgt, ctl, th = int(g["type"]), int(g["target"]), int(g["control"]), float(g["theta"])
            if t == 0:
                rc = 0
            elif t == 1: rc = L.gate_pauli_x(p, tgt)
            elif t == 2: rc = L.gate_pauli_y(p, tgt)
            elif t == 3: rc = L.gate_pauli_z(p, tgt)
            elif t == 4: rc = L.gate_hadamard(p, tgt)
            elif t == 5: rc = L.gate_s(p, tgt)
            elif t == 6: rc = L.gate_t(p, tgt)
            elif t == 7: rc = L.gate_rx(p, tgt, th)
            elif t == 8: rc = L.gate_ry(p, tgt, th)
            elif t == 9: rc = L.gate_rz(p, tgt, th)
            elif t == 10: rc = L.gate_cnot(p, ctl, tgt)
            elif t == 11:  # qgtl composition S . CNOT . Sdg
                rc = L.gate_s(p, tgt) or L.gate_cnot(p, ctl, tgt) or L.gate_s_dagger(p, tgt)
            elif t == 12: rc = L.gate_cz(p, ctl, tgt)
            elif t == 13: rc = L.gate_swap(p, ctl, tgt)
            elif t == 20: rc = L.gate_s_dagger(p, tgt)
            elif t == 21: rc = L.gate_t_dagger(p, tgt)
            elif t == 22: rc = L.gate_phase(p, tgt, th)
            elif t == 23: rc = L.gate_cphase(p, ctl, tgt, th)
            elif t == 24: rc = L.gate_crx(p, ctl, tgt, th)
            elif t == 25: rc = L.gate_cry(p, ctl, tgt, th)
            elif t == 26: rc = L.gate_crz(p, ctl, tgt, th)
            elif t == 27:  # ZZ = CNOT . RZ . CNOT (qaoa.c:745-753)
                rc = L.gate_cnot(p, ctl, tgt) or L.gate_rz(p, tgt, th) or L.gate_cnot(p, ctl, tgt)
            else:
                raise ValueError(f"gate type {t}")
            if rc:
                raise RuntimeError(f"reference gate {t} failed: {rc}")

    def probabilities(self) -> np.ndarray:
        out = np.empty(1 << self.n, dtype=np.float64)
        self.lib.measurement_probability_distribution(C.byref(self.s), _dp(out))
        return out

    def sample(self, uniforms) -> np.ndarray:
        u = np.ascontiguousarray(uniforms, dtype=np.float64)
        out = np.empty(len(u), dtype=np.uint64)
        self.lib.measurement_sample(C.byref(self.s), _u64p(out), len(u), _dp(u))
        return out

    def close(self):
        if self.s.amplitudes:
            self.lib.quantum_state_free(C.byref(self.s))
            self.s.amplitudes = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_qgtl_execute(n: int, gates, shots: int, seed: int, want_probs: bool = True):
    """moonlab_qgtl_execute through the reference's public API."""
    L = ref()
    c = L.moonlab_qgtl_circuit_create(n)
    for g in gates:
        t, tgt, ctl, th = int(g["type"]), int(g["target"]), int(g["control"]), float(g["theta"])
        par = C.c_double(th)
        rc = L.moonlab_qgtl_add_gate(c, t, tgt, ctl, C.byref(par) if t in (7, 8, 9) else None)
        if rc:
            raise RuntimeError(f"moonlab_qgtl_add_gate: {rc}")
    opts = QgtlOpts(shots, seed, 1 if want_probs else 0)
    res = QgtlResults()
    rc = L.moonlab_qgtl_execute(c, C.byref(opts), C.byref(res))
    L.moonlab_qgtl_circuit_free(c)
    if rc:
        raise RuntimeError(f"moonlab_qgtl_execute: {rc}")
    outs = np.ctypeslib.as_array(res.outcomes, shape=(shots,)).copy() if shots else np.empty(0, np.uint64)
    probs = np.ctypeslib.as_array(res.probabilities, shape=(1 << n,)).copy() if want_probs else None
    L.moonlab_qgtl_results_free(C.byref(res))
    return outs, probs


def ref_circuit_serialize(c) -> str:
    """moonlab_qgtl_circuit_serialize of a reference circuit handle."""
    L = ref()
    need = C.c_size_t()
    rc = L.moonlab_qgtl_circuit_serialize(c, None, 0, C.byref(need))
    if rc:
        raise RuntimeError(f"moonlab_qgtl_circuit_serialize: {rc}")
    buf = C.create_string_buffer(need.value + 1)
    rc = L.moonlab_qgtl_circuit_serialize(c, buf, len(buf), None)
    if rc:
        raise RuntimeError(f"moonlab_qgtl_circuit_serialize: {rc}")
    return buf.value.decode()


def ref_circuit_text(n: int, gates) -> str:
    """The reference's text for gate records (built with moonlab_qgtl_add_gate)."""
    L = ref()
    c = L.moonlab_qgtl_circuit_create(n)
    try:
        for g in gates:
            t, tgt, ctl, th = int(g["type"]), int(g["target"]), int(g["control"]), float(g["theta"])
            par = C.c_double(th)
            rc = L.moonlab_qgtl_add_gate(c, t, tgt, ctl, C.byref(par) if t in (7, 8, 9) else None)
            if rc:
                raise RuntimeError(f"moonlab_qgtl_add_gate: {rc}")
        return ref_circuit_serialize(c)
    finally:
        L.moonlab_qgtl_circuit_free(c)


def ref_circuit_roundtrip(raw: bytes, explicit_len: bool = True):
    """(status, re-serialized text or None) of moonlab_qgtl_circuit_deserialize."""
    L = ref()
    st = C.c_int(0)
    c = L.moonlab_qgtl_circuit_deserialize(raw, len(raw) if explicit_len else 0, C.byref(st))
    if not c:
        return st.value, None
    try:
        return st.value, ref_circuit_serialize(c)
    finally:
        L.moonlab_qgtl_circuit_free(c)


class RefSolver:
    """A vqe_solver_t built through the reference API: the hardware-efficient
    ansatz with `layers` layers, or ansatz=("uccsd", electrons) /
    ("symmetry", occupied, layers)."""

    def __init__(self, n: int, layers: int, paulis, coeffs, hf_reference: int = 0, ansatz=None):
        L = self.lib = ref()
        self.h = L.pauli_hamiltonian_create(n, len(paulis))
        for k, (ps, c) in enumerate(zip(paulis, coeffs)):
            if L.pauli_hamiltonian_add_term(self.h, float(c), ps.encode(), k):
                raise RuntimeError("pauli_hamiltonian_add_term")
        if hf_reference:
            # pauli_hamiltonian_t.hf_reference (vqe.h:127) sits after
            # num_qubits, num_terms, terms, nuclear_repulsion, molecule_name,
            # bond_distance: byte offset 48
            C.c_uint64.from_address(self.h + 48).value = hf_reference
        if ansatz is None:
            self.ans = L.vqe_create_hardware_efficient_ansatz(n, layers)
        elif ansatz[0] == "uccsd":
            self.ans = L.vqe_create_uccsd_ansatz(n, ansatz[1])
        elif ansatz[0] == "symmetry":
            self.ans = L.vqe_create_symmetry_preserving_ansatz(n, ansatz[1], ansatz[2])
        else:
            raise ValueError(ansatz)
        if not self.ans:
            raise RuntimeError(f"ansatz {ansatz} not created")
        self.opt = L.vqe_optimizer_create(2)  # any optimizer; vqe_solver_create needs one
        self.ctx = EntropyCtx(ENTROPY_FN(lambda ud, buf, sz: 0), None)
        self.solver = L.vqe_solver_create(self.h, self.ans, self.opt, C.byref(self.ctx))
        # vqe_ansatz_t.num_parameters (vqe.h:229-236): type (int, padded), num_qubits, num_layers, then it
        self.P = C.c_size_t.from_address(self.ans + 24).value
        if ansatz is None:
            assert self.P == 2 * n * layers

    def gradient(self, params) -> np.ndarray:
        p = np.ascontiguousarray(params, dtype=np.float64)
        g = np.empty(self.P, dtype=np.float64)
        rc = self.lib.moonlab_vqe_gradient(self.solver, _dp(p), _dp(g), self.P)
        if rc:
            raise RuntimeError(f"moonlab_vqe_gradient: {rc}")
        return g

    def _tensor(self, fn, params) -> np.ndarray:
        p = np.ascontiguousarray(params, dtype=np.float64)
        out = np.empty((self.P, self.P), dtype=np.float64)
        rc = fn(self.solver, _dp(p), _dp(out), self.P)
        if rc:
            raise RuntimeError(f"quantum geometry verb: {rc}")
        return out

    def qgt(self, params) -> np.ndarray:
        """moonlab_vqe_qgt: the metric g = Re Q."""
        return self._tensor(self.lib.moonlab_vqe_qgt, params)

    def berry_curvature(self, params) -> np.ndarray:
        """moonlab_vqe_berry_curvature: F = -2 Im Q."""
        return self._tensor(self.lib.moonlab_vqe_berry_curvature, params)

    def natural_gradient(self, params, gradient, regularization: float) -> np.ndarray:
        """moonlab_vqe_natural_gradient (the stable verb)."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        gr = np.ascontiguousarray(gradient, dtype=np.float64)
        out = np.empty(self.P, dtype=np.float64)
        rc = self.lib.moonlab_vqe_natural_gradient(self.solver, _dp(p), _dp(gr), regularization, _dp(out), self.P)
        if rc:
            raise RuntimeError(f"moonlab_vqe_natural_gradient: {rc}")
        return out

    def natural_gradient_direction(self, params, gradient, regularization: float) -> np.ndarray:
        p = np.ascontiguousarray(params, dtype=np.float64)
        gr = np.ascontiguousarray(gradient, dtype=np.float64)
        out = np.empty(self.P, dtype=np.float64)
        rc = self.lib.vqe_natural_gradient_direction(self.solver, _dp(p), _dp(gr), regularization, _dp(out))
        if rc:
            raise RuntimeError(f"vqe_natural_gradient_direction: {rc}")
        return out

    def close(self):
        if self.solver:
            self.lib.vqe_solver_free(self.solver)
            self.solver = None


def ref_vqe_gradient(n: int, layers: int, paulis, coeffs, params) -> np.ndarray:
    """moonlab_vqe_gradient on a HEA solver built through the reference API."""
    L = ref()
    h = L.pauli_hamiltonian_create(n, len(paulis))
    for k, (ps, c) in enumerate(zip(paulis, coeffs)):
        if L.pauli_hamiltonian_add_term(h, float(c), ps.encode(), k):
            raise RuntimeError("pauli_hamiltonian_add_term")
    ans = L.vqe_create_hardware_efficient_ansatz(n, layers)
    opt = L.vqe_optimizer_create(2)  # ADAM (any; vqe_solver_create needs one)
    ctx = EntropyCtx(ENTROPY_FN(lambda ud, buf, sz: 0), None)
    solver = L.vqe_solver_create(h, ans, opt, C.byref(ctx))
    P = 2 * n * layers
    p = np.ascontiguousarray(params, dtype=np.float64)
    g = np.empty(P, dtype=np.float64)
    rc = L.moonlab_vqe_gradient(solver, _dp(p), _dp(g), P)
    L.vqe_solver_free(solver)
    if rc:
        raise RuntimeError(f"moonlab_vqe_gradient: {rc}")
    return g
