"""The continuous-batching request loop (mlb_server_*).

Each request's outcomes are the same alone and in a concurrent mix (both
dtypes, bit-identical), complex128 outcomes equal the oracle's
moonlab_qgtl_execute restatement (pinned to the reference), requests that
arrive while a large one runs are admitted and finish before it, admission
holds the HBM budget, and the error paths report what they should."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from moonlab_b200 import _lib
from moonlab_b200.circuits import Request, brickwork, config_c5
from oracle import bindings as B


def test_request_stream_is_seeded():
    a, b = config_c5(num=50), config_c5(num=50)
    assert a == b
    assert all(10 <= r.n <= 28 and 10 <= r.depth <= 100 and 1 <= r.shots <= 4096 for r in a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))


def test_server_needs_a_device():
    from moonlab_b200.serving import _bind
    lib = _bind()
    cnt = C.c_int()
    if lib.mlb_device_count(C.byref(cnt)) == 0 and cnt.value > 0:
        pytest.skip("a device is present")
    h = C.c_void_p()
    assert lib.mlb_server_create(0, 0, 4, C.byref(h)) == -2


def _mix(num, seed=0x5E):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(num):
        n = int(rng.integers(10, 21))
        reqs.append(Request(i, 0.0, n, int(rng.integers(5, 30)), int(rng.integers(1, 600)),
                            int(rng.integers(0, 2)), int(rng.integers(1, 2**63))))
    return reqs


@pytest.mark.gpu
def test_same_alone_and_in_the_mix(gpu):
    from moonlab_b200.serving import Server, request_circuit
    reqs = _mix(40)
    circ = [request_circuit(r) for r in reqs]
    alone = []
    with Server(workers=1) as s:
        for r, g in zip(reqs, circ):
            t = s.submit(r.n, g, r.shots, r.seed, "c64" if r.dtype else "c128")
            alone.append(s.wait(t)[0])
    # all at once, 8 in flight, a budget that holds only a few 20-qubit states
    with Server(workers=8, hbm_budget=(16 << 20) * 4 + (8 << 20)) as s:
        tickets = [s.submit(r.n, g, r.shots, r.seed, "c64" if r.dtype else "c128") for r, g in zip(reqs, circ)]
        mixed = [s.wait(t)[0] for t in tickets]
        st = s.stats()
    assert st["peak_running"] > 1
    assert st["peak_reserved_bytes"] <= st["budget_bytes"]
    for a, b in zip(alone, mixed):
        assert np.array_equal(a, b)
    # complex128 against the oracle's moonlab_qgtl_execute (bit-exact)
    for r, g, out in zip(reqs, circ, mixed):
        if r.dtype == 0 and r.n <= 16:
            want = np.empty(r.shots, dtype=np.uint64)
            sv = B.to_svo(g)
            assert B.port().svo_qgtl_execute(r.n, sv, len(sv), r.shots, r.seed,
                                              want.ctypes.data_as(C.POINTER(C.c_uint64)), None) == 0
            assert np.array_equal(out, want)


@pytest.mark.gpu
def test_late_arrivals_overtake_a_long_request(gpu):
    from moonlab_b200.serving import Server
    with Server(workers=4) as s:
        big = s.submit(27, brickwork(27, 80, 1), 16, 7, "c128")
        small = [s.submit(12, brickwork(12, 10, 2 + i), 64, 9 + i, "c64") for i in range(6)]
        infos = [s.wait(t)[1] for t in small]
        _, binfo = s.wait(big)
    assert all(i["admit_s"] < binfo["done_s"] for i in infos)
    assert all(i["done_s"] < binfo["done_s"] for i in infos)


@pytest.mark.gpu
def test_budget_errors_and_timeouts(gpu):
    from moonlab_b200.serving import Server
    from moonlab_b200._lib import MlbError
    with Server(workers=1, hbm_budget=64 << 20) as s:
        with pytest.raises(MlbError):
            s.submit(26, brickwork(26, 1, 3), 1, 1)  # 1 GiB state > 64 MiB budget
        t1 = s.submit(20, brickwork(20, 60, 4), 1, 1)
        t2 = s.submit(20, brickwork(20, 60, 5), 1, 1)
        with pytest.raises(TimeoutError):
            s.wait(t2, timeout_ms=0)  # behind t1 on the single worker
        s.wait(t1)
        out, info = s.wait(t2)
        assert info["status"] == 0 and len(out) == 1
        assert s.stats()["completed"] == 2


@pytest.mark.gpu
def test_small_requests_share_launches(gpu):
    """Small circuits (<= 12 qubits c128, <= 13 c64) run many per launch;
    each one's outcomes equal its run alone and, for complex128, the
    oracle's moonlab_qgtl_execute bit for bit."""
    from moonlab_b200.serving import Server
    from test_fused_plan import mixed_circuit
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(150):
        dt = int(rng.integers(0, 2))
        n = int(rng.integers(3, 13 if dt == 0 else 14))
        g = mixed_circuit(n, int(rng.integers(2, 12)), 100 + i) if n >= 4 else brickwork(n, 6, 100 + i, 2)
        reqs.append((n, g, int(rng.integers(1, 700)), int(rng.integers(1, 2**62)), "c64" if dt else "c128"))
    alone = []
    with Server(workers=1) as s:
        for n, g, shots, seed, dt in reqs:
            alone.append(s.wait(s.submit(n, g, shots, seed, dt))[0])
    with Server(workers=2) as s:
        tickets = [s.submit(*r) for r in reqs]
        done = [s.wait(t) for t in tickets]
        st = s.stats()
    mixed = [d[0] for d in done]
    # a request's times are final when its result is: submit <= admit <= done
    for _, info in done:
        assert 0.0 <= info["submit_s"] <= info["admit_s"] <= info["done_s"]
    assert st["small_requests"] == len(reqs)
    assert st["small_batches"] < len(reqs)
    for a, b in zip(alone, mixed):
        assert np.array_equal(a, b)
    for (n, g, shots, seed, dt), out in zip(reqs, mixed):
        if dt == "c128":
            want = np.empty(shots, dtype=np.uint64)
            sv = B.to_svo(g)
            assert B.port().svo_qgtl_execute(n, sv, len(sv), shots, seed,
                                              want.ctypes.data_as(C.POINTER(C.c_uint64)), None) == 0
            assert np.array_equal(out, want)


@pytest.mark.gpu
def test_larger_complex128_requests_match_the_oracle(gpu):
    """Requests of the serving stream's shape up to 22 qubits (complex128):
    outcomes bit-identical to the oracle's moonlab_qgtl_execute restatement,
    alone and when they share the device with others."""
    from moonlab_b200.serving import Server, request_circuit
    reqs = [Request(i, 0.0, n, d, shots, 0, seed) for i, (n, d, shots, seed) in
            enumerate([(18, 30, 200, 0x5A1), (20, 16, 128, 0x5A2), (21, 12, 96, 0x5A3), (22, 10, 64, 0x5A4),
                       (22, 14, 33, 0x5A5)])]
    circ = [request_circuit(r) for r in reqs]
    with Server(workers=4) as s:
        tickets = [s.submit(r.n, g, r.shots, r.seed, "c128") for r, g in zip(reqs, circ)]
        mixed = [s.wait(t)[0] for t in tickets]
    with Server(workers=1) as s:
        alone = [s.wait(s.submit(r.n, g, r.shots, r.seed, "c128"))[0] for r, g in zip(reqs, circ)]
    for r, g, a, b in zip(reqs, circ, alone, mixed):
        assert np.array_equal(a, b)
        want = np.empty(r.shots, dtype=np.uint64)
        sv = B.to_svo(g)
        assert B.port().svo_qgtl_execute(r.n, sv, len(sv), r.shots, r.seed,
                                          want.ctypes.data_as(C.POINTER(C.c_uint64)), None) == 0
        assert np.array_equal(a, want)
