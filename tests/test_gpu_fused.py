"""The fused complex64 path on the GPU (tcgen05 tensor cores, split-bf16
products, FP32 accumulation) against (a) the numpy replay of its own plan
(test_fused_plan.replay: same blocks and bf16 operand images, FP64
amplitudes), which isolates the kernel, and (b) the oracle: fidelity
>= 1 - 1e-6 and the max amplitude error reported."""
from __future__ import annotations

import numpy as np
import pytest

from moonlab_b200 import StateVector
from moonlab_b200.circuits import brickwork
from moonlab_b200.statevector import fused_plan
from oracle import bindings as B
from test_fused_plan import mixed_circuit, replay

pytestmark = pytest.mark.gpu


def run_fused(n, g):
    sv = StateVector(n, "c64")
    sv.set_exec_mode("fused")
    sv.run(g)
    out = sv.amplitudes()
    st = sv.flush_stats()
    sv.close()
    return out.astype(np.complex128), st


@pytest.mark.parametrize("n,depth", [(13, 4), (14, 6), (16, 5), (18, 3)])
def test_fused_kernel_matches_plan_replay(gpu, n, depth):
    g = mixed_circuit(n, depth, 0xF0 + n)
    got, st = run_fused(n, g)
    init = np.zeros(1 << n, dtype=np.complex128)
    init[0] = 1
    want = replay(fused_plan(g, n), n, init)
    scale = np.abs(want).max()
    assert st["dense_blocks"] > 0
    assert np.abs(got - want).max() < 2e-4 * scale


@pytest.mark.parametrize("n,depth", [(16, 12), (20, 20)])
def test_fused_fidelity_vs_oracle(gpu, n, depth):
    g = brickwork(n, depth, 0xC2 + n, zz_every=4)
    got, _ = run_fused(n, g)
    want = B.port_run(n, g)
    fid = abs(np.vdot(want, got)) ** 2 / np.vdot(got, got).real
    err = np.abs(got - want).max()
    print(f"n={n} depth={depth}: fidelity 1-{1 - fid:.3e}, max amplitude error {err:.3e}")
    assert fid >= 1 - 1e-6
    assert err < 1e-3


def test_fused_mode_needs_complex64_and_13_qubits(gpu):
    from moonlab_b200._lib import MlbError
    with StateVector(14, "c128") as sv, pytest.raises(MlbError):
        sv.set_exec_mode("fused")
    with StateVector(12, "c64") as sv, pytest.raises(MlbError):
        sv.set_exec_mode("fused")
