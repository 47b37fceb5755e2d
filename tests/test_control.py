"""The control-plane front end (mlb_control_*): the reference control
server's request frames (src/control/control_plane.h:8-33,
control_plane.c:598-770) executed on the device loop.  Frame handling and
the error frames run on the CPU; CIRCUIT probabilities and SHOTS outcomes
are checked against the oracle on the GPU."""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np
import pytest

from moonlab_b200.circuits import brickwork
from moonlab_b200.scheduler import format_circuit_text
from moonlab_b200.serving import ControlFrontEnd
from oracle import bindings as B


def frame(verb: str, text: str) -> bytes:
    body = text.encode()
    return f"{verb} {len(body)}\n".encode() + body


@pytest.mark.parametrize("req,resp", [
    (b"HEALTH\n", b"OK alive\n"),
    (b"HEALTH", b"OK alive\n"),
    (b"HEALTH \n", b"ERR -404 unknown verb\n"),
    (b"HEALTHX\n", b"ERR -404 unknown verb\n"),
    (b"METRICS\n", b"ERR -404 unknown verb\n"),  # served by the transport, not here
    (b"CIRCUIT x\n", b"ERR -404 expected CIRCUIT <N>\n"),
    (b"SHOTS 5\n", b"ERR -404 expected SHOTS <shots> <bytes>\n"),
    (b"SHOTS 0 10\nNUM_QUBITS 1\n", b"ERR -401 shots out of range\n"),
    (b"SHOTS 1048577 10\n", b"ERR -401 shots out of range\n"),
    (b"CIRCUIT 0\n", b"ERR -401 body bytes out of range\n"),
    (b"CIRCUIT 4194305\n", b"ERR -401 body bytes out of range\n"),
    (b"CIRCUIT 40\nNUM_QUBITS 2\n", b"ERR -404 short body\n"),
    (b"CIRCUIT 13\nNUM_QUBITS 0\n", b"ERR -405 deserialize\n"),
    (b"CIRCUIT 14\nNUM_QUBITS 2\nX\n", b"ERR -405 deserialize\n"),
    (b"", b"ERR -404 empty frame\n"),
    (b"C" * 120, b"ERR -404 header too long\n"),
])
def test_frames_without_execution(req, resp):
    with ControlFrontEnd() as c:
        assert c.handle(req) == resp


def test_qubit_cap():
    text = "NUM_QUBITS 31\nH 30\n"
    with ControlFrontEnd() as c:  # default cap: 30, the reference's ceiling
        assert c.handle(frame("CIRCUIT", text)) == b"ERR -401 qubit count exceeds server cap\n"
    with ControlFrontEnd(max_qubits=8) as c:
        assert c.handle(frame("SHOTS 4", "NUM_QUBITS 9\nH 0\n")) == b"ERR -401 qubit count exceeds server cap\n"
    with pytest.raises(RuntimeError):
        ControlFrontEnd(max_qubits=34)


def split(resp: bytes):
    head, _, payload = resp.partition(b"\n")
    return head.decode(), payload


@pytest.mark.gpu
def test_circuit_probabilities_match_the_oracle(gpu):
    n = 12
    g = brickwork(n, 10, 0xC7)
    with ControlFrontEnd() as c:
        head, payload = split(c.handle(frame("CIRCUIT", format_circuit_text(n, g))))
    assert head == f"OK {1 << n}"
    got = np.frombuffer(payload, dtype="<f8")
    want = B.port_probabilities(B.port_run(n, g), rule=1)  # re*re + im*im
    assert got.size == want.size and np.abs(got - want).max() < 1e-12


@pytest.mark.gpu
def test_shots_match_moonlab_qgtl_execute(gpu):
    n, shots, seed = 10, 3000, 0x5EED
    g = brickwork(n, 8, 0xC8)
    with ControlFrontEnd(workers=4) as c:
        c.set_seed(seed)
        head, payload = split(c.handle(frame(f"SHOTS {shots}", format_circuit_text(n, g))))
    assert head == f"SAMPLES {shots}"
    got = np.frombuffer(payload, dtype="<u8")
    want = np.empty(shots, dtype=np.uint64)
    sv = B.to_svo(g)
    assert B.port().svo_qgtl_execute(n, sv, len(sv), shots, seed, want.ctypes.data_as(C.POINTER(C.c_uint64)),
                                     None) == 0
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_concurrent_requests(gpu):
    # many connection threads at once, as the reference's server runs them;
    # clock-seeded shots of a basis state are all the same bitstring
    texts = {q: f"NUM_QUBITS {q}\n" + "".join(f"X {t}\n" for t in range(0, q, 2)) for q in (6, 11, 15, 18)}
    results = {}

    with ControlFrontEnd(workers=4) as c:
        def one(k, q):
            results[k] = (q, c.handle(frame("SHOTS 64", texts[q])))

        ts = [threading.Thread(target=one, args=(k, q)) for k, q in enumerate(list(texts) * 4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        health = c.handle(b"HEALTH\n")
    assert health == b"OK alive\n"
    assert len(results) == 16
    for q, resp in results.values():
        head, payload = split(resp)
        assert head == "SAMPLES 64"
        want = sum(1 << t for t in range(0, q, 2))
        assert np.all(np.frombuffer(payload, dtype="<u8") == want)
