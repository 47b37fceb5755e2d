"""Generate tests/golden/c2_prefix_30q.npz: the reference's own results on a
30-qubit prefix of the 30-qubit depth-40 random circuit (seed 0xC2, a ZZ
layer every 4 layers).

The prefix is the first 4 layers (RX, RY, RZ on every qubit, then the CNOT
brickwork) plus the ZZ(theta) layer after layer 3: 447 gate records, 505
reference gate calls (ZZ = CNOT . RZ . CNOT, qaoa.c:745-753).  The state is
16 GiB, too large to store, so the fixture keeps what a test can compare
exactly:

* <Z_i> for all 30 qubits (measurement_expectation_z, measurement.c:428);
* the norm (sum of |a|^2 over the reference's amplitudes);
* 4096 amplitudes at seeded indices, and their probabilities from
  measurement_probability_distribution (measurement.c:140);
* 1024 outcomes of measurement_sample (measurement.c:551-601) for the
  seeded uniforms stored beside them.

Every value is computed by the reference library built from its sources
(oracle/Makefile -> oracle/_ref/liboracle.so, all host threads).  About ten
minutes on 8 cores and 33 GB of host memory:

    make -C oracle ref REF=<reference tree> && python tests/golden/gen_c2_prefix.py
"""
from __future__ import annotations

import ctypes as C
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO))

from moonlab_b200.circuits import SplitMix64, brickwork  # noqa: E402
from oracle import bindings as B  # noqa: E402

OUT = Path(__file__).resolve().parent / "c2_prefix_30q.npz"
N = 30
DEPTH = 40
SEED = 0xC2
PREFIX_LAYERS = 4
NUM_AMPS = 4096
NUM_SHOTS = 1024


def c2_prefix() -> np.ndarray:
    """The first PREFIX_LAYERS layers of the depth-40 circuit and the ZZ
    layer after them: angles are the depth-40 circuit's own (same stream)."""
    full = brickwork(N, DEPTH, SEED, zz_every=4)
    cnots_per_layer = [len(range(l % 2, N - 1, 2)) for l in range(PREFIX_LAYERS)]
    count = sum(3 * N + c for c in cnots_per_layer) + (N - 1)
    pre = full[:count]
    assert (pre["type"][-(N - 1):] == 27).all() and (pre["type"][:-(N - 1)] != 27).all()
    return pre


def main() -> None:
    L = B.ref()
    gates = c2_prefix()
    t0 = time.time()
    r = B.RefStateVector(N)
    r.run(gates)
    t_run = time.time() - t0
    a = np.frombuffer((C.c_double * (2 << N)).from_address(r.s.amplitudes), dtype=np.complex128)
    idx_rng = SplitMix64(0xC2A3B1)
    idx = np.unique(np.array([idx_rng.next() >> (64 - N) for _ in range(NUM_AMPS)], dtype=np.int64))
    amps = a[idx].copy()
    norm = float(np.sum(a.real * a.real + a.imag * a.imag))
    ez = np.array([L.measurement_expectation_z(C.byref(r.s), q) for q in range(N)])
    probs = r.probabilities()[idx].copy()
    u = SplitMix64(SEED ^ 0x5EED5EED).uniforms(NUM_SHOTS)
    outs = r.sample(u)
    r.close()
    np.savez_compressed(OUT, gates=gates, n=np.int32(N), amp_index=idx, amps=amps, probs=probs,
                        norm=np.float64(norm), ez=ez, uniforms=u, outcomes=outs)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes); {len(gates)} gates, reference run {t_run:.0f} s, "
          f"total {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
