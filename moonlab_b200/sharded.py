"""Sharded states: one n-qubit state split over 2^g ranks, one shard of
2^(n-g) amplitudes per rank, for states above one device's memory.

Reference: src/distributed/state_partition.{h,c} (the top g qubits are the
rank bits; partition_execute_exchange, state_partition.h:383) and
src/distributed/distributed_gates.c:241-290, :784-900 (a gate on a rank
qubit is a host-staged MPI exchange of the pair's amplitudes per gate).

Here a logical qubit is not tied to a physical bit: a layout maps logical
qubits to physical positions, positions 0..n-g-1 local to a shard and
n-g..n-1 the rank bits.  A gate whose non-diagonal targets are local runs
on each shard as it is, with its controls and diagonal keys on rank bits
resolved per rank (a control that a rank's bit fails drops the op there; a
diagonal key on a rank bit becomes a constant or a local diagonal).  A
target on a rank bit is first swapped with a local qubit: the two ranks of
each pair exchange the half-shard whose local bit differs from their rank
bit (one send/recv of 2^(n-g-1) amplitudes each way, into the same slots),
and the layout records the swap.  The local qubit chosen is the one whose
next use as a target is furthest ahead, so one swap serves many gates.

The local ops run on an executor: `EngineExecutor` keeps the shard in an
engine state on this rank's device (the tile kernels).  `ShardedState` runs
one shard per rank and exchanges through torch.distributed (NCCL send/recv
between devices); `LocalShards` holds all shards in one process and
exchanges by device-to-device copies.  Either way an exchange moves the
half-shard in chunks through one reusable staging buffer per direction, so
it never needs more than one chunk of extra memory (the reference's bounded
buffer_size exchange, distributed_gates.c:241-273).  `gather` returns the
whole state in logical qubit order.
"""
from __future__ import annotations

import numpy as np

from . import _lib

OP_1Q, OP_2Q, OP_DIAG1, OP_X, OP_SWAP, OP_ZZ, OP_PHASE = range(7)


def op_targets(o) -> list:
    """Non-diagonal targets of an op (they must be local to run)."""
    if o.kind in (OP_1Q, OP_X):
        return [o.target]
    if o.kind in (OP_2Q, OP_SWAP):
        return [o.target, o.target2]
    return []


class Layout:
    """Logical qubit -> physical position; positions >= n_loc are rank bits."""

    def __init__(self, n: int, g: int):
        if not 0 <= g < n:
            raise ValueError("need 0 <= rank bits < qubits")
        self.n, self.g, self.n_loc = n, g, n - g
        self.phys = list(range(n))
        self.logical = list(range(n))

    def is_local(self, q: int) -> bool:
        return self.phys[q] < self.n_loc

    def swap(self, j: int, l: int) -> None:
        """Exchange rank bit j with local position l."""
        G = self.n_loc + j
        a, b = self.logical[G], self.logical[l]
        self.phys[a], self.phys[b] = l, G
        self.logical[G], self.logical[l] = b, a


def plan(ops, n: int, g: int, lookahead: int = 512, start: Layout | None = None):
    """Steps for running ops on 2^g ranks from layout `start` (default: the
    identity): ("ops", phys, [op indices]) runs those ops with the layout
    phys, and ("swap", j, l) exchanges rank bit j with local position l.
    The steps depend only on the ops and the layout, so every rank takes the
    same exchanges.  Returns the steps and the final layout."""
    lay = Layout(n, g)
    if start is not None:
        lay.phys, lay.logical = list(start.phys), list(start.logical)
    steps, batch = [], []
    nxt = {}  # logical qubit -> indices where it is a target, in order
    for i, o in enumerate(ops):
        for q in op_targets(o):
            nxt.setdefault(q, []).append(i)
    ptr = {q: 0 for q in nxt}

    def next_use(q: int, i: int) -> int:
        uses = nxt.get(q, [])
        k = ptr.get(q, 0)
        while k < len(uses) and uses[k] < i:
            k += 1
        ptr[q] = k
        return uses[k] - i if k < len(uses) and uses[k] - i <= lookahead else lookahead + 1

    for i, o in enumerate(ops):
        tq = op_targets(o)
        for q in tq:
            if lay.is_local(q):
                continue
            if batch:
                steps.append(("ops", list(lay.phys), batch))
                batch = []
            best, best_score = None, -1
            for p in range(lay.n_loc):  # the local qubit needed as a target latest
                b = lay.logical[p]
                if b in tq:
                    continue
                score = next_use(b, i + 1)
                if score > best_score:
                    best, best_score = p, score
            if best is None:
                raise ValueError(f"op {i} has {len(tq)} targets but a shard has only {lay.n_loc} local "
                                 "qubits: need more local qubits than the widest op has targets")
            j = lay.phys[q] - lay.n_loc
            steps.append(("swap", j, best))
            lay.swap(j, best)
        batch.append(i)
    if batch:
        steps.append(("ops", list(lay.phys), batch))
    return steps, lay


def _const_op(c: complex, cmask: int):
    """amp *= c where the local controls cmask hold."""
    o = _lib.MlbOp()
    if cmask:
        o.kind, o.target, o.target2, o.cmask = OP_PHASE, -1, -1, cmask
        o.m[0], o.m[1] = c.real, c.imag
    else:  # a phase op needs a mask: the same factor on both halves of qubit 0
        o.kind, o.target, o.target2, o.cmask = OP_DIAG1, 0, -1, 0
        o.m[0], o.m[1], o.m[2], o.m[3] = c.real, c.imag, c.real, c.imag
    return o


def localize(o, phys, n_loc: int, rank: int):
    """The op as rank `rank` runs it on its shard (physical local positions),
    or None when its rank-bit conditions fail there."""
    def rbit(q):
        return (rank >> (phys[q] - n_loc)) & 1

    cm = 0
    for q in range(64):
        if o.cmask >> q & 1:
            if phys[q] >= n_loc:
                if not rbit(q):
                    return None
            else:
                cm |= 1 << phys[q]
    r = _lib.MlbOp.from_buffer_copy(o)
    r.cmask = cm
    if o.kind in (OP_1Q, OP_X, OP_2Q, OP_SWAP):
        r.target = phys[o.target]
        if o.kind in (OP_2Q, OP_SWAP):
            r.target2 = phys[o.target2]
        return r
    d0, d1 = complex(o.m[0], o.m[1]), complex(o.m[2], o.m[3])
    if o.kind == OP_PHASE:
        return r if cm else _const_op(d0, 0)
    if o.kind == OP_DIAG1:
        if phys[o.target] >= n_loc:
            return _const_op(d1 if rbit(o.target) else d0, cm)
        r.target = phys[o.target]
        return r
    if o.kind == OP_ZZ:  # d0 where the two bits are equal, d1 where they differ
        ga, gb = phys[o.target] >= n_loc, phys[o.target2] >= n_loc
        if ga and gb:
            return _const_op(d1 if rbit(o.target) ^ rbit(o.target2) else d0, cm)
        if ga or gb:
            v = rbit(o.target) if ga else rbit(o.target2)
            u = o.target2 if ga else o.target
            e0, e1 = (d1, d0) if v else (d0, d1)
            r.kind, r.target, r.target2 = OP_DIAG1, phys[u], -1
            r.m[0], r.m[1], r.m[2], r.m[3] = e0.real, e0.imag, e1.real, e1.imag
            return r
        r.target, r.target2 = phys[o.target], phys[o.target2]
        return r
    raise ValueError(f"op kind {o.kind} cannot be sharded")


DEFAULT_CHUNK = 1 << 24  # amplitudes per exchange chunk (256 MiB of complex128)


def half_view(shard, l: int, j: int, rank: int):
    """The half-shard that rank-bit j <-> local bit l moves off this rank: the
    slots whose local bit l differs from this rank's bit j, as an R x C
    strided view (C = 2^l contiguous amplitudes per row)."""
    a = (rank >> j) & 1
    n_half = shard.numel() // 2
    return shard.view(n_half >> l, 2, 1 << l)[:, 1 - a, :]


def chunks(rows: int, cols: int, chunk: int):
    """Row-major blocks (r0, r1, c0, c1) of at most `chunk` elements that
    cover a rows x cols view, the same sequence on every rank."""
    if chunk < 1:
        raise ValueError("chunk must be at least one amplitude")
    if cols <= chunk:
        step = max(1, chunk // cols)
        for r0 in range(0, rows, step):
            yield r0, min(rows, r0 + step), 0, cols
    else:
        for r in range(rows):
            for c0 in range(0, cols, chunk):
                yield r, r + 1, c0, min(cols, c0 + chunk)


class Staging:
    """The bounded staging an exchange goes through: one send and one receive
    buffer of `chunk` amplitudes, allocated on first use and reused, so an
    exchange never holds more than one chunk of extra memory per direction
    (the reference exchanges through a fixed buffer_size in chunks,
    distributed_gates.c:241-273)."""

    def __init__(self, chunk: int = DEFAULT_CHUNK):
        if chunk < 1:
            raise ValueError("chunk must be at least one amplitude")
        self.chunk = chunk
        self.send = self.recv = None

    def buffers(self, like):
        k = min(self.chunk, like.numel() // 2)
        if self.send is None or self.send.numel() < k or self.send.device != like.device:
            self.send = like.new_empty(k)
            self.recv = like.new_empty(k)
        return self.send, self.recv


def exchange_half(shard, l: int, j: int, rank: int, group=None, staging: Staging | None = None) -> None:
    """Rank-bit j <-> local bit l: swap the half-shard whose local bit l
    differs from this rank's bit j with the partner rank (rank ^ 2^j), slot
    for slot, one staging chunk at a time (send and receive on the same
    buffers for every chunk)."""
    import torch.distributed as dist
    staging = staging or Staging()
    partner = rank ^ (1 << j)
    if group is not None:
        partner = dist.get_global_rank(group, partner)
    view = half_view(shard, l, j, rank)
    send, recv = staging.buffers(shard)
    R, Cn = view.shape
    for r0, r1, c0, c1 in chunks(R, Cn, send.numel()):
        blk = view[r0:r1, c0:c1]
        k = blk.numel()
        s, r = send[:k].view(blk.shape), recv[:k].view(blk.shape)
        s.copy_(blk)
        ops = [dist.P2POp(dist.isend, send[:k], partner, group), dist.P2POp(dist.irecv, recv[:k], partner, group)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        blk.copy_(r)


def exchange_local(lo_shard, hi_shard, l: int, staging: Staging | None = None) -> None:
    """The same exchange between two shards held by one process (rank r with
    bit j = 0 and its partner r | 2^j, on one device or two): lo's half with
    local bit l = 1 swaps with hi's half with bit l = 0, one staging chunk at
    a time, as device-to-device copies."""
    staging = staging or Staging()
    va = half_view(lo_shard, l, 0, 0)
    vb = half_view(hi_shard, l, 0, 1)
    tmp, _ = staging.buffers(lo_shard)
    R, Cn = va.shape
    for r0, r1, c0, c1 in chunks(R, Cn, tmp.numel()):
        a, b = va[r0:r1, c0:c1], vb[r0:r1, c0:c1]
        t = tmp[:a.numel()].view(a.shape)
        t.copy_(a)
        a.copy_(b)
        b.copy_(t)


class EngineExecutor:
    """This rank's shard in an engine state (complex128) on `device`: local
    ops run as the state's tile passes; `shard` is a torch view of its
    device memory for the exchange."""

    def __init__(self, n_loc: int, device: int):
        import torch
        from .statevector import StateVector
        self.sv = StateVector(n_loc, "c128", device=device)
        self._lib = _lib.load()
        self.shard = torch.as_tensor(_DeviceView(self.sv.device_ptr(), 1 << n_loc),
                                     device=f"cuda:{device}")

    def apply(self, ops) -> None:
        if ops:
            arr = (_lib.MlbOp * len(ops))(*ops)
            _lib.check(self._lib.mlb_apply_ops(self.sv.handle, arr, len(ops)), "mlb_apply_ops")

    def sync(self) -> None:
        """Queued ops finished on the device (before an exchange reads the shard)."""
        self.sv.synchronize()

    def written(self) -> None:
        """Writes to `shard` through torch finished (before the state's stream reads it)."""
        import torch
        torch.cuda.synchronize(self.shard.device)

    def close(self) -> None:
        self.sv.close()


class _DeviceView:
    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<c16", "data": (ptr, False),
                                         "version": 3, "strides": None}


class ShardedState:
    """An n-qubit state over the ranks of `group` (a power of two), starting
    in |0...0>: rank 0's shard holds amplitude 0."""

    def __init__(self, n: int, executor, group=None, chunk: int = DEFAULT_CHUNK):
        import torch.distributed as dist
        self.ws = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        g = self.ws.bit_length() - 1
        if 1 << g != self.ws:
            raise ValueError("the number of ranks must be a power of two")
        self.n, self.g, self.n_loc = n, g, n - g
        self.group = group
        self.ex = executor
        self.layout = Layout(n, g)
        self.exchanges = 0
        self.staging = Staging(chunk)
        self.ex.sync()  # the executor's own initialisation has finished
        self.ex.shard.zero_()
        if self.rank == 0:
            self.ex.shard[0] = 1.0
        self.ex.written()

    def run_ops(self, ops) -> None:
        """Apply engine ops (mlb_op_t records on logical qubits) in order."""
        ops = list(ops)
        steps, _ = plan(ops, self.n, self.g, start=self.layout)
        for st in steps:
            if st[0] == "ops":
                _, phys, idx = st
                local = [localize(ops[i], phys, self.n_loc, self.rank) for i in idx]
                self.ex.apply([o for o in local if o is not None])
            else:
                _, j, l = st
                self.ex.sync()
                exchange_half(self.ex.shard, l, j, self.rank, self.group, self.staging)
                self.ex.written()
                self.layout.swap(j, l)
                self.exchanges += 1
        self.ex.sync()

    def run(self, gates) -> None:
        """Apply gate records (the QGTL enum and its extensions)."""
        from .statevector import gates_to_ops
        self.run_ops(gates_to_ops(gates, self.n))

    def gather(self):
        """The whole state in logical qubit order, on every rank (numpy)."""
        import torch
        import torch.distributed as dist
        loc = self.ex.shard.detach()
        parts = [torch.empty_like(loc) for _ in range(self.ws)]
        dist.all_gather(parts, loc, group=self.group)
        full = torch.cat([p.cpu() for p in parts]).numpy()  # physical index = rank << n_loc | local
        n = self.n
        src = [n - 1 - self.layout.phys[n - 1 - k] for k in range(n)]
        return np.ascontiguousarray(full.reshape([2] * n).transpose(src)).reshape(-1)


class LocalShards:
    """An n-qubit state as 2^g shards held by one process: one executor per
    shard, on one device or spread over this node's devices.  The same plan,
    per-shard op rewrite and half-shard exchanges as ShardedState, with each
    pair's exchange done as chunked device-to-device copies instead of
    torch.distributed messages."""

    def __init__(self, n: int, executors, chunk: int = DEFAULT_CHUNK):
        W = len(executors)
        g = W.bit_length() - 1
        if W < 1 or 1 << g != W:
            raise ValueError("the number of shards must be a power of two")
        self.n, self.g, self.n_loc = n, g, n - g
        self.ex = list(executors)
        self.layout = Layout(n, g)
        self.exchanges = 0
        self.staging = Staging(chunk)
        for r, e in enumerate(self.ex):
            e.sync()
            e.shard.zero_()
            if r == 0:
                e.shard[0] = 1.0
            e.written()

    def run_ops(self, ops) -> None:
        """Apply engine ops (mlb_op_t records on logical qubits) in order."""
        ops = list(ops)
        steps, _ = plan(ops, self.n, self.g, start=self.layout)
        for st in steps:
            if st[0] == "ops":
                _, phys, idx = st
                for r, e in enumerate(self.ex):
                    local = [localize(ops[i], phys, self.n_loc, r) for i in idx]
                    e.apply([o for o in local if o is not None])
            else:
                _, j, l = st
                for e in self.ex:
                    e.sync()
                for r in range(len(self.ex)):
                    if not (r >> j) & 1:
                        exchange_local(self.ex[r].shard, self.ex[r | (1 << j)].shard, l, self.staging)
                for e in self.ex:
                    e.written()
                self.layout.swap(j, l)
                self.exchanges += 1
        for e in self.ex:
            e.sync()

    def run(self, gates) -> None:
        """Apply gate records (the QGTL enum and its extensions)."""
        from .statevector import gates_to_ops
        self.run_ops(gates_to_ops(gates, self.n))

    def gather(self):
        """The whole state in logical qubit order (numpy)."""
        import torch
        full = torch.cat([e.shard.detach().cpu() for e in self.ex]).numpy()
        n = self.n
        src = [n - 1 - self.layout.phys[n - 1 - k] for k in range(n)]
        return np.ascontiguousarray(full.reshape([2] * n).transpose(src)).reshape(-1)
