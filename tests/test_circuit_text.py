"""The "moonlab-circuit v1" text format (mlb_circuit_parse_text /
mlb_circuit_format_text) against the reference's own serializer and
deserializer (src/applications/moonlab_qgtl_backend.c:319-506): the committed
fixture tests/golden/circuit_text.json (made by tests/golden/gen_golden.py from
the reference library) and, where the reference library is built, a fuzz run
compared case by case."""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from moonlab_b200 import _lib
from moonlab_b200.circuits import GATE_DTYPE
from moonlab_b200.scheduler import format_circuit_text, parse_circuit_text
from oracle import bindings as B

INVALID_ARG, NOT_SUPPORTED = -6, -9  # MLB_ERR_INVALID_ARG, MLB_ERR_NOT_SUPPORTED (moonlab_b200.h)
FIXTURE = json.loads((Path(__file__).parent / "golden" / "circuit_text.json").read_text())


def fixture_gates():
    g = np.zeros(len(FIXTURE["gates"]), dtype=GATE_DTYPE)
    for i, (t, tgt, ctl, th) in enumerate(FIXTURE["gates"]):
        g[i] = (t, tgt, ctl if 10 <= t <= 13 else -1, 0, float.fromhex(th))
    return g


def parse_raw(raw: bytes, length: int):
    """(status, num_qubits, gates) through the C ABI with an explicit length."""
    lib = _lib.load()
    nq, n = C.c_uint32(), C.c_size_t()
    st = lib.mlb_circuit_parse_text(raw, length, C.byref(nq), None, 0, C.byref(n))
    if st:
        return st, None, None
    g = np.zeros(n.value, dtype=GATE_DTYPE)
    st = lib.mlb_circuit_parse_text(raw, length, C.byref(nq), g.ctypes.data_as(C.c_void_p), n.value, C.byref(n))
    return st, int(nq.value), g


def test_format_matches_the_reference_serializer():
    assert format_circuit_text(FIXTURE["num_qubits"], fixture_gates()) == FIXTURE["text"]


def test_parse_gives_the_serialized_records():
    n, g = parse_circuit_text(FIXTURE["text"])
    want = fixture_gates()
    assert n == FIXTURE["num_qubits"]
    assert np.array_equal(g["type"], want["type"])
    assert np.array_equal(g["target"], want["target"])
    assert np.array_equal(g["control"], want["control"])
    # theta round-trips bit for bit (%.17g), -0.0 and the smallest subnormal included
    assert np.array_equal(g["theta"].view(np.uint64), want["theta"].view(np.uint64))


@pytest.mark.parametrize("case", FIXTURE["cases"], ids=lambda c: repr(c["text"][:40]))
def test_edge_cases_match_the_reference_deserializer(case):
    raw = case["text"].encode()
    st, n, g = parse_raw(raw, len(raw))
    if case["status"] != 0:
        assert st == INVALID_ARG
    else:
        assert st == 0
        assert format_circuit_text(n, g) == case["reserialized"]


def test_length_rules():
    text = b"NUM_QUBITS 3\nH 0\nCNOT 1 0\n"
    st, n, g = parse_raw(text, 0)  # length 0: a NUL-terminated string
    assert st == 0 and n == 3 and len(g) == 2
    st, _, _ = parse_raw(text + b"\0H 1\n", len(text) + 5)  # a NUL inside the declared extent
    assert st == INVALID_ARG
    st, n, g = parse_raw(text + b"H 2\n", len(text))  # bytes past the extent are not read
    assert st == 0 and len(g) == 2


def test_buffer_contracts():
    lib = _lib.load()
    raw = FIXTURE["text"].encode()
    nq, n = C.c_uint32(), C.c_size_t()
    assert lib.mlb_circuit_parse_text(raw, len(raw), C.byref(nq), None, 0, C.byref(n)) == 0
    total = n.value
    small = np.zeros(total - 1, dtype=GATE_DTYPE)
    assert lib.mlb_circuit_parse_text(raw, len(raw), C.byref(nq), small.ctypes.data_as(C.c_void_p), total - 1,
                                      C.byref(n)) == INVALID_ARG
    assert n.value == total
    g = fixture_gates()
    w = C.c_size_t()
    assert lib.mlb_circuit_format_text(10, g.ctypes.data_as(C.c_void_p), len(g), None, 0, C.byref(w)) == 0
    assert w.value == len(raw)
    buf = C.create_string_buffer(w.value)  # one byte short of text + NUL
    assert lib.mlb_circuit_format_text(10, g.ctypes.data_as(C.c_void_p), len(g), buf, len(buf),
                                       C.byref(w)) == INVALID_ARG
    assert w.value == len(raw) + 1
    zz = np.zeros(1, dtype=GATE_DTYPE)
    zz[0] = (27, 1, 0, 0, 0.5)  # ZZ(theta) has no name in the text format
    assert lib.mlb_circuit_format_text(4, zz.ctypes.data_as(C.c_void_p), 1, None, 0, C.byref(w)) == NOT_SUPPORTED


def mutate(rng, text: str) -> str:
    lines = text.split("\n")
    for _ in range(int(rng.integers(1, 4))):
        i = int(rng.integers(0, len(lines)))
        op = int(rng.integers(0, 9))
        s = lines[i]
        if op == 0 and s:
            j = int(rng.integers(0, len(s)))
            lines[i] = s[:j] + s[j + 1:]
        elif op == 1:
            j = int(rng.integers(0, len(s) + 1))
            lines[i] = s[:j] + str(rng.choice(list(" \t\r#-+.0123456789exXnNiIaAfF,"))) + s[j:]
        elif op == 2:
            lines.insert(i, str(rng.choice(["", "# c", "  ", "NUM_QUBITS 5", "H 9", "CNOT 3 3", "RX 1 nan"])))
        elif op == 3:
            del lines[i]
        elif op == 4:
            toks = s.split(" ")
            if len(toks) > 1:
                toks[int(rng.integers(1, len(toks)))] = str(int(rng.integers(-3, 14)))
                lines[i] = " ".join(toks)
        elif op == 5:
            toks = s.split(" ")
            toks[0] = str(rng.choice(["I", "X", "Y", "Z", "H", "S", "T", "RX", "RY", "RZ", "CNOT", "CY", "CZ",
                                      "SWAP", "rx", "CX", "U3", "HH"]))
            lines[i] = " ".join(toks)
        elif op == 6:
            lines[i] = " " * int(rng.integers(0, 4)) + s + " " * int(rng.integers(0, 4))
        elif op == 7:
            lines[i] = s + " " + str(rng.choice(["extra", "1", "0.5", "1e", "0x", "inf"]))
        else:
            lines[i] = s.replace(" ", "  ")
    return "\n".join(lines)


@pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")
def test_fuzzed_texts_match_the_reference():
    rng = np.random.default_rng(0x7E47)
    base = "# moonlab-circuit v1\nNUM_QUBITS 10\n" + "\n".join(FIXTURE["text"].split("\n")[2:40]) + "\n"
    for _ in range(600):
        t = mutate(rng, base)
        raw = t.encode()
        ref_st, ref_back = B.ref_circuit_roundtrip(raw)
        st, n, g = parse_raw(raw, len(raw))
        assert (st == 0) == (ref_st == 0), repr(t)
        if st == 0:
            assert format_circuit_text(n, g) == ref_back, repr(t)


@pytest.mark.gpu
def test_parsed_circuit_runs_like_the_oracle(gpu):
    from moonlab_b200 import StateVector
    n, g = parse_circuit_text(FIXTURE["text"])
    with StateVector(n, "c128") as sv:
        sv.run(g)
        got = sv.amplitudes()
    want = B.port_run(n, g)
    assert np.abs(got - want).max() < 1e-12
