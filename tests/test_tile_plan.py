"""The tile-pass planner on the host (mlb_tile_plan): every plan, replayed in
numpy in its execution order, gives the circuit's state, and keeps the
constraints the tile kernel relies on (non-diagonal targets inside the
pass's tile and, in a gate-by-gate segment, among its register bits).
Brickwork, QAOA and random circuits of every gate kind, complex128 (dense
segments, conditioning limits, filled high slots, lifted parity phases) and
complex64."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from moonlab_b200 import _lib, gates_to_ops
from moonlab_b200.circuits import GATE_DTYPE, brickwork, qaoa_circuit

OP_1Q, OP_2Q, OP_DIAG1, OP_X, OP_SWAP, OP_ZZ, OP_PHASE = range(7)
_IDX = {}


C128_TILE_BITS = 12  # complex128 tiles: 2 contiguous low qubits + 10 chosen high ones


def apply_op(a, n, o):
    """mlb_op_t semantics (moonlab_b200.h) on a numpy state, in place."""
    idx = _IDX.setdefault(n, np.arange(1 << n, dtype=np.uint64))
    mm = np.ctypeslib.as_array(o.m)
    c = mm[0::2] + 1j * mm[1::2]
    cm = np.uint64(o.cmask)
    sel = (idx & cm) == cm
    t, t2 = int(o.target), int(o.target2)
    if o.kind in (OP_1Q, OP_X, OP_DIAG1):
        tb = np.uint64(1 << t)
        i0 = idx[sel & ((idx & tb) == 0)]
        i1 = i0 | tb
        a0, a1 = a[i0].copy(), a[i1].copy()
        if o.kind == OP_X:
            a[i0], a[i1] = a1, a0
        elif o.kind == OP_DIAG1:
            a[i0], a[i1] = c[0] * a0, c[1] * a1
        else:
            a[i0], a[i1] = c[0] * a0 + c[1] * a1, c[2] * a0 + c[3] * a1
    elif o.kind in (OP_2Q, OP_SWAP):
        b0, b1 = np.uint64(1 << t), np.uint64(1 << t2)
        base = idx[sel & ((idx & (b0 | b1)) == 0)]
        ii = [base, base | b0, base | b1, base | b0 | b1]
        x = [a[i].copy() for i in ii]
        if o.kind == OP_SWAP:
            a[ii[1]], a[ii[2]] = x[2], x[1]
        else:
            M = c[:16].reshape(4, 4)
            for r in range(4):
                a[ii[r]] = sum(M[r, k] * x[k] for k in range(4))
    elif o.kind == OP_ZZ:
        par = ((idx >> np.uint64(t)) ^ (idx >> np.uint64(t2))) & np.uint64(1)
        a[sel] *= np.where(par == 0, c[0], c[1])[sel]
    elif o.kind == OP_PHASE:
        a[sel] *= c[0]
    else:
        raise AssertionError(f"op kind {o.kind}")


def replay(n, ops, seed=5):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    a /= np.linalg.norm(a)
    for o in ops:
        apply_op(a, n, o)
    return a


def tile_plan(ops, n, dtype, fuse=1):
    lib = _lib.load()
    np_, ns, no = C.c_size_t(), C.c_size_t(), C.c_size_t()
    _lib.check(lib.mlb_tile_plan(ops, len(ops), n, dtype, fuse, None, C.byref(np_), None, C.byref(ns), None,
                                 C.byref(no)), "mlb_tile_plan")
    passes = (_lib.MlbTilePass * np_.value)()
    segs = (_lib.MlbTileSegment * ns.value)()
    planned = (_lib.MlbOp * no.value)()
    _lib.check(lib.mlb_tile_plan(ops, len(ops), n, dtype, fuse, passes, C.byref(np_), segs, C.byref(ns), planned,
                                 C.byref(no)), "mlb_tile_plan")
    return list(passes), list(segs), planned


def check_structure(n, passes, segs, planned, dtype):
    """Pass and segment constraints of the tile kernel; returns the segment modes."""
    covered = []
    modes = []
    for p in passes:
        L, H = p.num_low, p.num_high
        assert L + H <= 13
        high = list(p.high[:H])
        pos = {q: q for q in range(L)}
        pos.update({q: L + i for i, q in enumerate(high)})
        assert len(pos) == L + H  # distinct tile qubits
        for s in segs[p.seg_begin:p.seg_begin + p.num_segments]:
            covered.append((s.op_begin, s.op_end))
            modes.append(s.mode)
            ops = planned[s.op_begin:s.op_end]
            regs = set(s.bits[:s.nbits])
            for o in ops:
                tq = {OP_1Q: [o.target], OP_X: [o.target], OP_2Q: [o.target, o.target2],
                      OP_SWAP: [o.target, o.target2]}.get(o.kind, [])
                assert all(q in pos for q in tq), "target outside the tile"
                if s.mode == 0:
                    assert all(pos[q] in regs for q in tq), "target outside the register bits"
            if s.mode == 1:
                assert len(ops) == 1 and ops[0].kind == OP_2Q
            if s.mode == 2:
                assert dtype == _lib.MLB_C128 and L + H == C128_TILE_BITS and s.nbits == 4
    # the segments cover the execution order once, in order
    flat = [i for b, e in covered for i in range(b, e)]
    assert flat == list(range(len(planned)))
    return modes


def random_gates(n, count, seed):
    rng = np.random.default_rng(seed)
    types = list(range(14)) + list(range(20, 28))
    g = np.zeros(count, dtype=GATE_DTYPE)
    for i in range(count):
        t = int(rng.choice(types))
        q = rng.permutation(n)
        two = t in (10, 11, 12, 13) or t >= 23
        g[i] = (t, int(q[0]), int(q[1]) if two else -1, 0, float(rng.uniform(-np.pi, np.pi)))
    return g


CIRCUITS = {
    "brickwork14": (14, lambda: brickwork(14, 12, 0xB1, zz_every=3)),
    "brickwork16": (16, lambda: brickwork(16, 8, 0xB2, zz_every=4)),
    "qaoa14": (14, lambda: qaoa_circuit(14, 2, 0x9A)),
    "random14": (14, lambda: random_gates(14, 400, 0xA11)),
    "random13": (13, lambda: random_gates(13, 300, 0xA12)),
    "random9": (9, lambda: random_gates(9, 200, 0xA13)),
}


@pytest.mark.parametrize("dtype", [_lib.MLB_C128, _lib.MLB_C64], ids=["c128", "c64"])
@pytest.mark.parametrize("name", list(CIRCUITS))
def test_plan_replays_the_circuit(name, dtype):
    n, make = CIRCUITS[name]
    g = make()
    ops = gates_to_ops(g, n)
    passes, segs, planned = tile_plan(ops, n, dtype)
    check_structure(n, passes, segs, planned, dtype)
    want = replay(n, ops)
    got = replay(n, planned)
    assert np.abs(got - want).max() < 1e-12
    # the plan is the one a flush runs: same pass count as mlb_plan_ops
    st = _lib.MlbFlushStats()
    _lib.check(_lib.load().mlb_plan_ops(ops, len(ops), n, dtype, 1, C.byref(st)), "mlb_plan_ops")
    assert st.passes == len(passes) and st.segments == len(segs) and st.ops == len(planned)
    if dtype == _lib.MLB_C128:
        assert st.dense_blocks == sum(1 for s in segs if s.mode == 2)


@pytest.mark.parametrize("name", ["brickwork14", "brickwork16", "qaoa14"])
def test_complex128_segments_all_run_dense(name):
    n, make = CIRCUITS[name]
    ops = gates_to_ops(make(), n)
    passes, segs, planned = tile_plan(ops, n, _lib.MLB_C128)
    assert all(s.mode == 2 for s in segs)
    assert all(p.num_low + p.num_high == C128_TILE_BITS for p in passes)  # high slots filled


def test_unfused_plan_keeps_every_op():
    n = 14
    ops = gates_to_ops(CIRCUITS["random14"][1](), n)
    passes, segs, planned = tile_plan(ops, n, _lib.MLB_C64, fuse=0)
    assert len(planned) == len(ops)
    check_structure(n, passes, segs, planned, _lib.MLB_C64)
    assert np.abs(replay(n, planned) - replay(n, ops)).max() < 1e-12


def test_buffer_contract():
    lib = _lib.load()
    n = 14
    ops = gates_to_ops(CIRCUITS["brickwork14"][1](), n)
    np_, ns, no = C.c_size_t(), C.c_size_t(), C.c_size_t()
    _lib.check(lib.mlb_tile_plan(ops, len(ops), n, 0, 1, None, C.byref(np_), None, C.byref(ns), None,
                                 C.byref(no)), "mlb_tile_plan")
    want = (np_.value, ns.value, no.value)
    short = C.c_size_t(ns.value - 1)
    segs = (_lib.MlbTileSegment * max(1, short.value))()
    rc = lib.mlb_tile_plan(ops, len(ops), n, 0, 1, None, C.byref(np_), segs, C.byref(short), None, C.byref(no))
    assert rc == -6 and (np_.value, short.value, no.value) == want  # MLB_ERR_INVALID_ARG, sizes reported
