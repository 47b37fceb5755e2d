"""Sharded states (moonlab_b200.sharded): the swap planner, the per-rank op
rewrite and the half-shard exchange, checked against a whole-state numpy
replay.  First all ranks simulated in one process (the exchange done on
numpy shards), then real gloo ranks on the CPU through torch.distributed,
with a numpy executor standing in for the device engine."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from moonlab_b200 import gates_to_ops
from moonlab_b200 import sharded as S
from moonlab_b200.circuits import GATE_DTYPE, brickwork, qaoa_circuit
from test_tile_plan import apply_op, random_gates

ROOT = Path(__file__).resolve().parents[1]
TOL = 1e-12


def to_logical(full, n, phys):
    src = [n - 1 - phys[n - 1 - k] for k in range(n)]
    return np.ascontiguousarray(full.reshape([2] * n).transpose(src)).reshape(-1)


def whole_state(n, ops):
    a = np.zeros(1 << n, complex)
    a[0] = 1
    for o in ops:
        apply_op(a, n, o)
    return a


def simulate(n, g, ops):
    """Every rank in one process; returns the logical state and the exchanges."""
    steps, lay = S.plan(ops, n, g)
    W, nl = 1 << g, n - g
    shards = [np.zeros(1 << nl, complex) for _ in range(W)]
    shards[0][0] = 1
    swaps = 0
    for st in steps:
        if st[0] == "ops":
            _, phys, idx = st
            for o in (ops[i] for i in idx):
                assert all(phys[q] < nl for q in S.op_targets(o)), "target on a rank bit"
            for r in range(W):
                for i in idx:
                    lo = S.localize(ops[i], phys, nl, r)
                    if lo is not None:
                        apply_op(shards[r], nl, lo)
        else:
            _, j, l = st
            swaps += 1
            for r in range(W):
                if not (r >> j) & 1:
                    p = r | (1 << j)
                    A, B = shards[r].reshape(-1, 2, 1 << l), shards[p].reshape(-1, 2, 1 << l)
                    tmp = A[:, 1, :].copy()
                    A[:, 1, :] = B[:, 0, :]
                    B[:, 0, :] = tmp
    return to_logical(np.concatenate(shards), n, lay.phys), swaps


CIRCUITS = {
    "brickwork": lambda n: brickwork(n, 10, 0x5A, zz_every=3),
    "qaoa": lambda n: qaoa_circuit(n, 2, 0x5B),
    "random": lambda n: random_gates(n, 300, 0x5C + n),
}


@pytest.mark.parametrize("g", [1, 2, 3])
@pytest.mark.parametrize("name", list(CIRCUITS))
def test_simulated_ranks_match_the_whole_state(name, g):
    n = 9
    ops = list(gates_to_ops(CIRCUITS[name](n), n))
    got, swaps = simulate(n, g, ops)
    assert np.abs(got - whole_state(n, ops)).max() < TOL
    assert swaps > 0


def test_swaps_are_amortised():
    # brickwork targets every qubit in every layer, so each layer must move
    # the g qubits on rank bits out at least once: 2 x 20 swaps at best here;
    # one exchange per gate on a rank qubit (the reference's way) takes 140
    n, g, depth = 12, 2, 20
    ops = list(gates_to_ops(brickwork(n, depth, 0x5D), n))
    steps, _ = S.plan(ops, n, g)
    swaps = sum(1 for s in steps if s[0] == "swap")
    per_gate = sum(1 for o in ops for q in S.op_targets(o) if q >= n - g)
    assert per_gate == 140
    assert g * depth <= swaps <= g * depth + 4


def test_rank_bit_conditions():
    # a control on a rank bit drops the op on ranks whose bit is 0; diagonal
    # keys on rank bits become constants or local diagonals
    n, g = 6, 2
    lay = S.Layout(n, g)
    o = gates_to_ops(np.array([(10, 1, 5, 0, 0.0)], dtype=GATE_DTYPE), n)[0]  # CNOT 5 -> 1
    assert S.localize(o, lay.phys, n - g, rank=0) is None
    lo = S.localize(o, lay.phys, n - g, rank=2)  # rank bit 1 = qubit 5 set
    assert lo is not None and lo.target == 1 and lo.cmask == 0
    zz = gates_to_ops(np.array([(27, 2, 4, 0, 0.7)], dtype=GATE_DTYPE), n)[0]
    for r in range(4):
        lz = S.localize(zz, lay.phys, n - g, r)
        assert lz.kind == S.OP_DIAG1 and lz.target == 2


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class NumpyExecutor:
    """Stands in for the device engine on CPU ranks: the shard is a CPU
    torch tensor and local ops run through the numpy op applier."""

    def __init__(self, n_loc: int):
        import torch
        self.n_loc = n_loc
        self.shard = torch.zeros(1 << n_loc, dtype=torch.complex128)

    def apply(self, ops):
        a = self.shard.numpy()
        for o in ops:
            apply_op(a, self.n_loc, o)

    def sync(self):
        pass

    def written(self):
        pass


@pytest.mark.parametrize("rows,cols,chunk", [(1, 1, 1), (8, 4, 5), (8, 4, 4), (3, 16, 5), (2, 64, 64), (5, 1, 3)])
def test_chunks_cover_the_view_once(rows, cols, chunk):
    seen = np.zeros((rows, cols), int)
    for r0, r1, c0, c1 in S.chunks(rows, cols, chunk):
        assert (r1 - r0) * (c1 - c0) <= chunk
        seen[r0:r1, c0:c1] += 1
    assert (seen == 1).all()


def test_planner_rejects_too_few_local_qubits():
    # one local qubit cannot host a SWAP whose other target is a rank bit
    n, g = 2, 1
    ops = list(gates_to_ops(np.array([(13, 1, 0, 0, 0.0)], dtype=GATE_DTYPE), n))
    with pytest.raises(ValueError, match="local qubits"):
        S.plan(ops, n, g)


@pytest.mark.parametrize("g,chunk", [(1, 3), (2, 16), (3, 1 << 20)])
@pytest.mark.parametrize("name", list(CIRCUITS))
def test_local_shards_match_the_whole_state(name, g, chunk):
    # all shards in one process, exchanged in chunks of `chunk` amplitudes
    n = 9
    gates = CIRCUITS[name](n)
    st = S.LocalShards(n, [NumpyExecutor(n - g) for _ in range(1 << g)], chunk=chunk)
    half = len(gates) // 2
    st.run(gates[:half])
    st.run(gates[half:])
    want = whole_state(n, list(gates_to_ops(gates, n)))
    assert np.abs(st.gather() - want).max() < TOL
    assert st.exchanges > 0
    assert st.staging.send.numel() == min(chunk, 1 << (n - g - 1))  # the only extra memory


def _rank(rank, ws, port, n, name, q, chunk=S.DEFAULT_CHUNK):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        g = ws.bit_length() - 1
        st = S.ShardedState(n, NumpyExecutor(n - g), chunk=chunk)
        gates = CIRCUITS[name](n)
        half = len(gates) // 2
        st.run(gates[:half])  # two calls: the second starts from a permuted layout
        st.run(gates[half:])
        full = st.gather()
        q.put((rank, full, st.exchanges))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,name,chunk", [(2, "brickwork", S.DEFAULT_CHUNK), (2, "random", 7),
                                           (4, "qaoa", 32), (4, "random", S.DEFAULT_CHUNK)])
def test_gloo_ranks_match_the_whole_state(ws, name, chunk):
    import torch.multiprocessing as mp
    n = 9
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, n, name, q, chunk)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(ws)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    want = whole_state(n, list(gates_to_ops(CIRCUITS[name](n), n)))
    for _, full, ex in res:
        assert np.abs(full - want).max() < TOL
        assert ex > 0
    assert len({ex for _, _, ex in res}) == 1  # every rank took the same exchanges
