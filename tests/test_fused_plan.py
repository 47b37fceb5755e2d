"""The fused complex64 path's host plan (dense <= 5-qubit blocks, tile
passes, bf16 hi/lo operand images), replayed in numpy FP64 and compared with
the oracle: a planning error (wrong block order, tile bits, padding or
operand layout) shows as an O(1) amplitude error, the bf16 split of U' alone
as ~1e-5.  The GPU kernel is checked against the same replay in
test_gpu_fused.py."""
from __future__ import annotations

import numpy as np
import pytest

from moonlab_b200.circuits import GATE_DTYPE, brickwork
from moonlab_b200.statevector import fused_plan
from oracle import bindings as B


def sw128_table():
    n = np.arange(64)[:, None]
    k = np.arange(64)[None, :]
    lin = (n // 8) * 1024 + (n % 8) * 128 + 2 * k
    return (lin ^ ((n % 8) << 4)) // 2  # bf16 element index


SW = sw128_table()


def bf16(u16):
    return (u16.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def block_unitary(img):
    """U (32x32 complex) from a 16 KiB operand image: hi + lo of U'."""
    raw = np.frombuffer(img.tobytes(), dtype=np.uint16)
    up = bf16(raw[:4096][SW]) + bf16(raw[4096:][SW])  # U'[n][k]
    return up[:32, :32] + 1j * up[32:, :32]


def deposit(v, bits):
    out = np.zeros_like(v)
    for i, b in enumerate(bits):
        out |= ((v >> i) & 1) << b
    return out


def tile_bits(p):
    """Qubits in a pass's tile: its low qubits plus its chosen high ones."""
    return p["num_low"] + len(p["hbits"])


def replay(plan, n, state):
    st = state.astype(np.complex128).copy()
    imgs = plan["images"].reshape(-1, 16384)
    for p in plan["passes"]:
        hb, L, tb = p["hbits"], p["num_low"], tile_bits(p)
        e = np.arange(1 << tb, dtype=np.int64)
        rest = [q for q in range(n) if q >= L and q not in hb]
        t = np.arange(p["num_tiles"], dtype=np.int64)
        G = deposit(t, rest)[:, None] | deposit(e, list(range(L)) + hb)[None, :]
        T = st[G]
        for blk in plan["blocks"][p["block_begin"]:p["block_begin"] + p["num_blocks"]]:
            idx = deposit(np.arange(1 << (tb - 5), dtype=np.int64), blk["rows"][:tb - 5])[:, None] | \
                deposit(np.arange(32, dtype=np.int64), blk["pos"])[None, :]
            U = block_unitary(imgs[blk["image"]])
            T[:, idx] = T[:, idx] @ U.T
        st[G] = T
    return st


def mixed_circuit(n, depth, seed):
    g = list(brickwork(n, depth, seed, zz_every=3))
    rng = np.random.default_rng(seed)
    for _ in range(12):  # controlled and 2-qubit gates on arbitrary pairs
        a, b = rng.choice(n, 2, replace=False)
        t = int(rng.choice([12, 13, 23, 24, 25, 26]))
        g.append((t, int(b), int(a), 0, float(rng.uniform(0, 6.28))))
    return np.array(g, dtype=GATE_DTYPE)


@pytest.mark.parametrize("n,depth", [(13, 4), (14, 6), (16, 5), (18, 3)])
def test_fused_plan_replays_the_circuit(n, depth):
    g = mixed_circuit(n, depth, 0xF0 + n)
    plan = fused_plan(g, n)
    assert len(plan["blocks"]) > 0 and all(p["num_blocks"] > 0 for p in plan["passes"])
    tb = tile_bits(plan["passes"][0])
    assert tb in (12, 13)
    for b in plan["blocks"]:
        assert sorted(b["pos"] + b["rows"][:tb - 5]) == list(range(tb))
    for p in plan["passes"]:
        L = p["num_low"]
        assert tile_bits(p) == tb
        assert len(set(p["hbits"])) == tb - L and min(p["hbits"]) >= L and max(p["hbits"]) < n
    init = np.zeros(1 << n, dtype=np.complex128)
    init[0] = 1
    got = replay(plan, n, init)
    want = B.port_run(n, g)
    fid = abs(np.vdot(want, got)) ** 2 / np.vdot(got, got).real
    assert np.abs(got - want).max() < 5e-4
    assert fid > 1 - 1e-7


def test_fused_plan_rejects_wide_ops_and_small_states():
    from moonlab_b200._lib import MlbError
    with pytest.raises(MlbError):
        fused_plan(brickwork(11, 2, 1), 11)
