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


def test_fused_mode_falls_back_to_tile_passes(gpu):
    """complex128 states refuse the fused mode; a complex64 state smaller
    than one tile (11 qubits), and an op on more than 5 qubits inside a fused
    circuit, run as tile passes in order with the fused blocks."""
    from moonlab_b200._lib import MlbError
    with StateVector(14, "c128") as sv, pytest.raises(MlbError):
        sv.set_exec_mode("fused")
    g11 = brickwork(11, 6, 3)
    got, st = run_fused(11, g11)
    assert st["dense_blocks"] == 0
    assert np.abs(got - B.port_run(11, g11)).max() < 1e-5
    n = 16
    with StateVector(n, "c64") as sv:
        sv.set_exec_mode("fused")
        g = brickwork(n, 4, 8)
        sv.run(g[: len(g) // 2])
        sv.mcx([0, 3, 7, 9, 12], 15)  # 6 qubits: a tile pass between fused runs
        sv.run(g[len(g) // 2:])
        got = sv.amplitudes().astype(np.complex128)
        st = sv.flush_stats()
    a = B.port_run(n, g[: len(g) // 2])
    idx = np.arange(1 << n)
    ctrl = (1 << 0) | (1 << 3) | (1 << 7) | (1 << 9) | (1 << 12)
    sel = (idx & ctrl) == ctrl
    b = a.copy()
    b[sel] = a[idx[sel] ^ (1 << 15)]
    want = B.port_run_from(n, g[len(g) // 2:], b)
    assert st["dense_blocks"] > 0
    assert np.abs(got - want).max() < 1e-5


def test_bounded_wait_reports_timeout_and_the_state_recovers(gpu):
    """The fused kernel's mbarrier waits are bounded: with CTA 0's first
    operand-image copy withheld (mlb_test_fused_skip_copy) its waits run out
    (20 ms each, no copy and no MMA in flight), the synchronize reports
    MLB_ERR_TIMEOUT, and the same state then reruns the circuit correctly."""
    from moonlab_b200 import _lib
    lib = _lib.load()
    n = 16
    g = brickwork(n, 6, 0x7AB, zz_every=3)
    want = B.port_run(n, g)
    with StateVector(n, "c64") as sv:
        sv.set_exec_mode("fused")
        assert lib.mlb_test_fused_skip_copy(sv.handle) == 0
        sv.run(g)
        assert lib.mlb_flush(sv.handle) == 0
        assert lib.mlb_synchronize(sv.handle) == -7  # MLB_ERR_TIMEOUT
        sv.reset()
        sv.run(g)
        got = sv.amplitudes().astype(np.complex128)
    fid = abs(np.vdot(want, got)) ** 2 / np.vdot(got, got).real
    assert fid >= 1 - 1e-6
