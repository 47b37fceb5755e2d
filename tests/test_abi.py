"""C-ABI surface checks that need no GPU: the library loads, exports every
function the public headers declare, reports the absence of a device
cleanly, and plans circuits on the host."""
from __future__ import annotations

import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

from moonlab_b200 import _lib, gates_to_ops
from moonlab_b200.circuits import GATE_DTYPE, brickwork, config_c1, config_c2, qaoa_circuit

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"#[^\n]*", "", text)
        text = re.sub(r"typedef[^;]*;", "", text)
        for stmt in text.split(";"):
            m = re.search(r"\b([A-Za-z_]\w*)\s*\([^()]*\)\s*$", stmt.strip())
            if m and m.group(1) not in ("if", "while", "sizeof", "enum", "struct"):
                names.add(m.group(1))
    return sorted(names)


def test_headers_declare_functions():
    names = header_functions()
    assert "mlb_state_create" in names and "quantum_state_create_gpu" in names
    assert len(names) > 60


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_status_strings():
    lib = _lib.load()
    assert lib.mlb_status_string(0) == b"ok"
    assert lib.mlb_status_string(-4) == b"invalid qubit"


def _has_gpu():
    cnt = C.c_int()
    return _lib.load().mlb_device_count(C.byref(cnt)) == 0 and cnt.value > 0


def test_no_device_is_reported_not_faked():
    if _has_gpu():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = C.c_void_p()
    rc = lib.mlb_state_create(10, 0, 0, C.byref(h))
    assert rc == -2 and not h.value  # MLB_ERR_NO_DEVICE, no state
    qs = C.POINTER(_lib.QuantumState)()
    assert lib.quantum_state_create_gpu(10, C.byref(qs)) == -7  # QS_ERROR_NOT_SUPPORTED
    assert not qs
    assert lib.moonlab_cuda_runtime_probe_discrete() in (0, -2)
    v = C.c_double(-1.0)
    assert lib.mlb_fp64_tensor_peak(0, C.byref(v)) == -2 and v.value == -1.0  # no probe figure made up


def test_gate_matrices_match_host_libm():
    th = 0.7312
    g = np.array([(7, 0, -1, 0, th), (8, 0, -1, 0, th), (9, 0, -1, 0, th), (6, 0, -1, 0, 0.0)],
                 dtype=GATE_DTYPE)
    ops = gates_to_ops(g, 1)
    c, s = math.cos(th / 2.0), math.sin(th / 2.0)
    assert list(ops[0].m[:8]) == [c, 0.0, 0.0, -s, 0.0, -s, c, 0.0]            # gates.c:392-395
    assert list(ops[1].m[:8]) == [c, 0.0, -s, 0.0, s, 0.0, c, 0.0]             # gates.c:438-440
    p0, p1 = complex(math.cos(-th / 2), math.sin(-th / 2)), complex(math.cos(th / 2), math.sin(th / 2))
    assert list(ops[2].m[:8]) == [p0.real, p0.imag, 0, 0, 0, 0, p1.real, p1.imag]  # gates.c:488-494
    t = complex(math.cos(math.pi / 4), math.sin(math.pi / 4))
    assert list(ops[3].m[:8]) == [1, 0, 0, 0, 0, 0, t.real, t.imag]


def test_invalid_gate_records_are_rejected():
    lib = _lib.load()
    bad = np.array([(10, 3, 3, 0, 0.0)], dtype=GATE_DTYPE)  # control == target
    cnt = C.c_size_t()
    rc = lib.mlb_gates_to_ops(bad.ctypes.data_as(C.POINTER(_lib.MlbGate)), 1, 5, None, C.byref(cnt))
    assert rc == -4
    bad = np.array([(7, 9, -1, 0, 0.1)], dtype=GATE_DTYPE)  # target outside the register
    rc = lib.mlb_gates_to_ops(bad.ctypes.data_as(C.POINTER(_lib.MlbGate)), 1, 5, None, C.byref(cnt))
    assert rc == -4


def plan(gates, n, dtype=0, fuse=1):
    lib = _lib.load()
    ops = gates_to_ops(gates, n)
    st = _lib.MlbFlushStats()
    _lib.check(lib.mlb_plan_ops(ops, len(ops), n, dtype, fuse, C.byref(st)), "mlb_plan_ops")
    return st


def test_planner_groups_the_brickwork_workloads():
    g1, _ = config_c1()
    st = plan(g1, 20)
    assert st.passes <= 20 and st.ops == 572      # 1390 gates, 1q runs fused
    g2, _ = config_c2()
    st = plan(g2, 30)
    assert st.passes <= 80                         # vs 4470 sweeps gate by gate
    assert st.bytes_moved == st.passes * 2 * 16 * (1 << 30)
    assert st.dense_amps == st.dense_blocks << 30  # planned for a dense state: every tile
    # c128: 12-bit tiles (2 contiguous low qubits), a pass's short trailing
    # segment deferred to the next pass: a few more passes, fewer dense segments
    assert st.passes <= 66 and st.segments <= 150
    # every register segment runs as a dense matrix (segments close before
    # their conditioning qubits outgrow one; full tiles)
    assert st.dense_blocks == st.segments
    for n in (16, 22, 26):
        st = plan(brickwork(n, 40, 0xC2, zz_every=4), n)
        assert st.dense_blocks == st.segments
    st64 = plan(g2, 30, dtype=1)
    assert st64.passes <= 65                       # c64: 5 contiguous low qubits per tile


def test_cnot_diagonal_cnot_is_lifted_to_one_zz():
    # QAOA's cost layer as the reference writes it: each CNOT . RZ . CNOT
    # becomes one parity-phase op; H and the RX mixer stay single ops
    g = qaoa_circuit(16, 3, 0x9A0A)
    edges = int((g["type"] == 9).sum()) // 3
    st = plan(g, 16)
    assert st.ops == 16 + 3 * (edges + 16)
    st0 = plan(g, 16, fuse=0)
    assert st0.ops == len(g)
    assert st.passes <= st0.passes
    # a controlled diagonal, or different controls, is left alone
    h = np.array([(10, 3, 1, 0, 0.0), (9, 3, -1, 0, 0.7), (10, 3, 2, 0, 0.0)], dtype=GATE_DTYPE)
    assert plan(h, 6).ops == 3


def test_planner_small_state_single_tile():
    # the whole 10-qubit state is one tile: passes only split the op program
    # into shared-memory-sized chunks (160 ops)
    st = plan(brickwork(10, 50, 7), 10)
    assert st.passes == -(-st.ops // 160)
    st = plan(brickwork(10, 5, 7), 10)
    assert st.passes == 1


def test_adjoint_problem_needs_a_device_and_valid_terms():
    lib = _lib.load()
    h = C.c_void_p()
    x = (C.c_uint64 * 1)(1 << 9)
    z = (C.c_uint64 * 1)(0)
    c = (C.c_double * 1)(1.0)
    # term outside a 4-qubit register is rejected before any device work
    assert lib.mlb_hea_create(4, 2, 0, 1, x, z, c, 0, 0, C.byref(h)) == -4
    if not _has_gpu():
        x[0] = 1
        assert lib.mlb_hea_create(4, 2, 0, 1, x, z, c, 0, 0, C.byref(h)) == -2
