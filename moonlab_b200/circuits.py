"""Seeded synthetic workloads: the random circuits, VQE problems and request
streams the engine is measured and checked on.

Random numbers come from splitmix64 in the increment form of the
reference's oracle corpus (tests/oracle/oracle_common.h:58-64); uniforms are
u = (x >> 11) * 2^-53; angles are 2 pi u; Gaussians use Box-Muller on two
successive uniforms.  Draw order is layer-major, then qubit-major, then
(RX, RY, RZ).  Gate records use the QGTL gate numbering
(moonlab_qgtl_backend.h:57-72) plus ZZ = 27.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

GATE_I, GATE_X, GATE_Y, GATE_Z, GATE_H, GATE_S, GATE_T = 0, 1, 2, 3, 4, 5, 6
GATE_RX, GATE_RY, GATE_RZ, GATE_CNOT, GATE_CY, GATE_CZ, GATE_SWAP = 7, 8, 9, 10, 11, 12, 13
GATE_ZZ = 27

MASK64 = (1 << 64) - 1
GAMMA = 0x9E3779B97F4A7C15

# numpy structured dtype matching mlb_gate_t {int32 type, target, control, reserved; double theta}
GATE_DTYPE = np.dtype([("type", "<i4"), ("target", "<i4"), ("control", "<i4"),
                       ("reserved", "<i4"), ("theta", "<f8")])


class SplitMix64:
    """splitmix64 with the golden-ratio increment (oracle_common.h:58-64)."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next(self) -> int:
        self.state = (self.state + GAMMA) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)

    def uniforms(self, k: int) -> np.ndarray:
        """The next k uniform() values at once (same sequence)."""
        if k <= 0:
            return np.empty(0, dtype=np.float64)
        z = np.uint64(self.state) + np.arange(1, k + 1, dtype=np.uint64) * np.uint64(GAMMA)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
        self.state = (self.state + k * GAMMA) & MASK64
        return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def gauss(self) -> float:
        u1 = self.uniform()
        u2 = self.uniform()
        u1 = u1 if u1 > 0.0 else 2.0 ** -53
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def splitmix64_finalizer(x: int) -> int:
    """The scheduler's worker-seed mix (scheduler.c:143-149), constants as there."""
    x &= MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D49BB133111EBB) & MASK64
    return x ^ (x >> 31)


def brickwork(n: int, depth: int, seed: int, zz_every: int = 0) -> np.ndarray:
    """Random brickwork circuit: per layer RX, RY, RZ on every qubit with
    angles U[0, 2pi), then CNOT(q, q+1) for q = (layer mod 2), step 2.  With
    zz_every = k > 0, after every layer l with (l + 1) mod k == 0 a ZZ(theta)
    on every neighbour pair (q, q+1), theta ~ U[0, 2pi).  Angles are drawn
    from SplitMix64(seed) in gate order."""
    zz_layers = [l for l in range(depth) if zz_every and (l + 1) % zz_every == 0]
    u = SplitMix64(seed).uniforms(3 * n * depth + len(zz_layers) * max(n - 1, 0))
    layers = []
    pos = 0
    qs = np.arange(n, dtype=np.int32)
    for layer in range(depth):
        rot = np.zeros(3 * n, dtype=GATE_DTYPE)
        rot["type"] = np.tile(np.array([GATE_RX, GATE_RY, GATE_RZ], dtype=np.int32), n)
        rot["target"] = np.repeat(qs, 3)
        rot["control"] = -1
        rot["theta"] = 2.0 * math.pi * u[pos:pos + 3 * n]
        pos += 3 * n
        layers.append(rot)
        c = np.arange(layer % 2, n - 1, 2, dtype=np.int32)
        cx = np.zeros(len(c), dtype=GATE_DTYPE)
        cx["type"] = GATE_CNOT
        cx["target"] = c + 1  # control q, target q+1
        cx["control"] = c
        layers.append(cx)
        if zz_every and (layer + 1) % zz_every == 0 and n > 1:
            zz = np.zeros(n - 1, dtype=GATE_DTYPE)
            zz["type"] = GATE_ZZ
            zz["target"] = qs[1:]
            zz["control"] = qs[:-1]
            zz["theta"] = 2.0 * math.pi * u[pos:pos + n - 1]
            pos += n - 1
            layers.append(zz)
    return np.concatenate(layers) if layers else np.zeros(0, dtype=GATE_DTYPE)


def qaoa_circuit(n: int, layers: int, seed: int, density: float = 0.3) -> np.ndarray:
    """QAOA on a random Ising graph, written the way the reference's solver
    applies it (src/algorithms/qaoa.c:594-602 cost layer, mixer after it):
    H on every qubit, then per layer CNOT(i, j) . RZ(j, 2 gamma J_ij) . CNOT(i, j)
    for every edge i < j and RX(q, 2 beta) on every qubit.  Edges (probability
    `density`), couplings U[-1.5, 1.5) and angles U[0, pi) from SplitMix64(seed)."""
    u = SplitMix64(seed)
    edges, J = [], []
    for i in range(n):
        for j in range(i + 1, n):
            if u.uniform() < density:
                edges.append((i, j))
                J.append(3.0 * u.uniform() - 1.5)
    recs = [(GATE_H, q, -1, 0, 0.0) for q in range(n)]
    for _ in range(layers):
        gamma, beta = math.pi * u.uniform(), math.pi * u.uniform()
        for (i, j), jij in zip(edges, J):
            recs += [(GATE_CNOT, j, i, 0, 0.0), (GATE_RZ, j, -1, 0, 2.0 * gamma * jij), (GATE_CNOT, j, i, 0, 0.0)]
        recs += [(GATE_RX, q, -1, 0, 2.0 * beta) for q in range(n)]
    return np.array(recs, dtype=GATE_DTYPE)


def config_c1(n: int = 20, depth: int = 20):
    """20-qubit depth-20 brickwork from |0..0>, 1024 shot uniforms."""
    gates = brickwork(n, depth, 0xC1)
    shots = SplitMix64(0xC1 ^ 0x5EED5EED).uniforms(1024)
    return gates, shots


def config_c2(n: int = 30, depth: int = 40):
    """30-qubit depth-40 brickwork with a ZZ layer every 4 layers."""
    gates = brickwork(n, depth, 0xC2, zz_every=4)
    shots = SplitMix64(0xC2 ^ 0x5EED5EED).uniforms(1024)
    return gates, shots


def config_c3(n: int, depth: int = 20):
    return brickwork(n, depth, 0xC3 ^ n)


@dataclass
class VQEProblem:
    n: int
    layers: int
    xmasks: np.ndarray   # uint64 [T]
    zmasks: np.ndarray   # uint64 [T]
    coeffs: np.ndarray   # float64 [T]
    paulis: list         # Pauli strings, char per qubit (index = qubit)
    params: np.ndarray   # float64 [B, P]


def config_c4(n: int = 20, layers: int = 8, batch: int = 256, num_terms: int | None = None,
              seed: int = 0xC4) -> VQEProblem:
    """HEA VQE problem: 4N random 2-local Pauli strings on distinct uniform
    pairs with N(0,1) coefficients; parameter vectors U[-pi, pi]."""
    rng = SplitMix64(seed)
    T = 4 * n if num_terms is None else num_terms
    xs, zs, cs, ps = [], [], [], []
    used = set()
    num_pairs = n * (n - 1) // 2
    while len(xs) < T:
        a = int(rng.uniform() * n)
        b = int(rng.uniform() * n)
        if len(used) == num_pairs:  # more terms than pairs: pairs repeat
            used.clear()
        if a == b or (min(a, b), max(a, b)) in used:
            continue
        used.add((min(a, b), max(a, b)))
        pa = "XYZ"[int(rng.uniform() * 3)]
        pb = "XYZ"[int(rng.uniform() * 3)]
        s = ["I"] * n
        s[a], s[b] = pa, pb
        x = z = 0
        for q, c in ((a, pa), (b, pb)):
            if c in "XY":
                x |= 1 << q
            if c in "YZ":
                z |= 1 << q
        xs.append(x)
        zs.append(z)
        cs.append(rng.gauss())
        ps.append("".join(s))
    P = 2 * n * layers
    params = np.array([[(2.0 * rng.uniform() - 1.0) * math.pi for _ in range(P)] for _ in range(batch)],
                      dtype=np.float64)
    return VQEProblem(n, layers, np.array(xs, dtype=np.uint64), np.array(zs, dtype=np.uint64),
                      np.array(cs, dtype=np.float64), ps, params)


@dataclass
class Request:
    rid: int
    arrival: float
    n: int
    depth: int
    shots: int
    dtype: int  # 0 complex128, 1 complex64
    seed: int


def config_c5(num: int = 10000, rate: float = 200.0, n_lo: int = 10, n_hi: int = 28,
              d_lo: int = 10, d_hi: int = 100, s_hi: int = 4096, seed: int = 0xC5) -> list:
    """Poisson request stream: qubits U{n_lo..n_hi}, depth U{d_lo..d_hi},
    shots U{1..s_hi}, dtype 50/50; per-request seed splitmix64(0xC5 ^ id)."""
    rng = SplitMix64(seed)
    t = 0.0
    out = []
    for rid in range(num):
        u = rng.uniform()
        t += -math.log(1.0 - u) / rate
        n = n_lo + int(rng.uniform() * (n_hi - n_lo + 1))
        d = d_lo + int(rng.uniform() * (d_hi - d_lo + 1))
        s = 1 + int(rng.uniform() * s_hi)
        dt = 1 if rng.uniform() < 0.5 else 0
        out.append(Request(rid, t, n, d, s, dt, splitmix64_finalizer(0xC5 ^ rid)))
    return out
