"""The persistent request loop for small circuits (mlb_mailbox_*).

One long-running launch serves posted requests: complex128 outcomes equal
the oracle's moonlab_qgtl_execute restatement bit for bit and complex64
outcomes equal the batch launch's (mlb_server_*); the loop's bounded wait
ends an idle launch with MLB_ERR_TIMEOUT and the next submit relaunches it;
a full ring, oversized requests and unknown tickets are refused."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

from moonlab_b200 import _lib
from moonlab_b200.circuits import brickwork
from oracle import bindings as B


def _requests(num, dtype, seed):
    from test_fused_plan import mixed_circuit
    rng = np.random.default_rng(seed)
    top = 13 if dtype == "c128" else 14
    out = []
    for i in range(num):
        n = int(rng.integers(3, top))
        g = mixed_circuit(n, int(rng.integers(2, 12)), 300 + i) if n >= 4 else brickwork(n, 6, 300 + i, 2)
        out.append((n, g, int(rng.integers(1, 900)), int(rng.integers(1, 2**62))))
    return out


def _run(mb, reqs, window=40):
    """Submit with at most `window` tickets outstanding; outcomes in order."""
    tickets, outs = [], [None] * len(reqs)
    for i, (n, g, shots, seed) in enumerate(reqs):
        if len(tickets) == window:
            j, t = tickets.pop(0)
            outs[j] = mb.wait(t)
        tickets.append((i, mb.submit(n, g, shots, seed)))
    for j, t in tickets:
        outs[j] = mb.wait(t)
    return outs


def test_mailbox_needs_a_device():
    from moonlab_b200.serving import MlbMailboxConfig, _bind
    lib = _bind()
    cnt = C.c_int()
    if lib.mlb_device_count(C.byref(cnt)) == 0 and cnt.value > 0:
        pytest.skip("a device is present")
    h = C.c_void_p()
    cfg = MlbMailboxConfig(_lib.MLB_C128, 0, 0, 0, 0, 0, 0.0)
    assert lib.mlb_mailbox_create(C.byref(cfg), C.byref(h)) == -2


@pytest.mark.gpu
def test_complex128_outcomes_match_the_oracle(gpu):
    from moonlab_b200.serving import Mailbox
    reqs = _requests(120, "c128", 21)
    with Mailbox("c128", ctas=8) as mb:
        outs = _run(mb, reqs)
        st = mb.stats()
    assert st["submitted"] == st["completed"] == len(reqs)
    for (n, g, shots, seed), out in zip(reqs, outs):
        want = np.empty(shots, dtype=np.uint64)
        sv = B.to_svo(g)
        assert B.port().svo_qgtl_execute(n, sv, len(sv), shots, seed,
                                          want.ctypes.data_as(C.POINTER(C.c_uint64)), None) == 0
        assert np.array_equal(out, want)


@pytest.mark.gpu
def test_complex64_outcomes_match_the_batch_launch(gpu):
    from moonlab_b200.serving import Mailbox, Server
    reqs = _requests(80, "c64", 22)
    with Mailbox("c64", ctas=4, slots=16) as mb:
        outs = _run(mb, reqs, window=12)
    with Server(workers=2) as s:
        tickets = [s.submit(n, g, shots, seed, "c64") for n, g, shots, seed in reqs]
        want = [s.wait(t)[0] for t in tickets]
    for a, b in zip(outs, want):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_idle_loop_ends_with_timeout_and_relaunches(gpu):
    from moonlab_b200.serving import Mailbox
    reqs = _requests(6, "c128", 23)
    with Mailbox("c128", ctas=2, idle_ms=20.0) as mb:
        first = _run(mb, reqs[:3])
        time.sleep(0.3)  # the loop's bounded wait runs out: the launch ends
        st = mb.stats()
        assert st["running"] == 0 and st["launches"] == 1 and st["idle_exits"] == 1
        second = _run(mb, reqs[3:])  # relaunched by the submit
        st = mb.stats()
        assert st["launches"] >= 2 and st["completed"] == 6
    for (n, g, shots, seed), out in zip(reqs, first + second):
        want = np.empty(shots, dtype=np.uint64)
        sv = B.to_svo(g)
        assert B.port().svo_qgtl_execute(n, sv, len(sv), shots, seed,
                                          want.ctypes.data_as(C.POINTER(C.c_uint64)), None) == 0
        assert np.array_equal(out, want)


@pytest.mark.gpu
def test_full_ring_and_limits_are_refused(gpu):
    from moonlab_b200.serving import Mailbox
    g = brickwork(8, 4, 7, 2)
    with Mailbox("c128", ctas=2, slots=4, max_shots=64) as mb:
        tickets = [mb.submit(8, g, 16, 100 + k) for k in range(4)]
        with pytest.raises(_lib.MlbError) as e:
            mb.submit(8, g, 16, 5)
        assert e.value.status == -8                      # MLB_ERR_BUSY: every slot holds a ticket
        with pytest.raises(_lib.MlbError) as e:
            mb.submit(8, g, 65, 5)
        assert e.value.status == -6                      # more shots than a slot holds
        with pytest.raises(_lib.MlbError) as e:
            mb.submit(13, brickwork(13, 2, 7, 2), 4, 5)
        assert e.value.status == -5                      # larger than a block's shared memory
        outs = [mb.wait(t) for t in tickets]
        assert all(len(o) == 16 for o in outs)
        assert mb.submit(8, g, 16, 5) >= 4             # slots free again
        rc = mb._lib.mlb_mailbox_wait(mb._h, 12345, 0, None, 0)
        assert rc == -6                                 # unknown ticket
