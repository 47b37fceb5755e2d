"""The 30-qubit depth-40 workload and the capacity limits on the device.

* Against the reference itself: a 447-gate prefix of the 30-qubit circuit
  (first 4 layers and the ZZ layer after them), run by the reference library
  into tests/golden/c2_prefix_30q.npz (tests/golden/gen_c2_prefix.py: <Z_i>,
  the norm, 4096 amplitudes at seeded indices, 1024 measurement_sample
  outcomes).  The engine's complex128 path with dense segments (its default)
  must give every stored amplitude to 1e-12, <Z_i> to 1e-12 (summed as the
  reference sums it; 1e-10 from the one-pass reduction) and the outcomes bit
  for bit.
* The whole depth-40 circuit: dense segments against gate-by-gate segments
  (engine against engine, 1e-12 per amplitude; the oracle cannot hold a
  30-qubit state in the time a test has), and the fused complex64 path
  against the complex128 result (fidelity >= 1 - 1e-6).
* Capacity: 33 qubits complex128 and 34 qubits complex64 (128 GiB each):
  the norm after a depth-20 circuit, and at 32 qubits complex64 against
  complex128 (fidelity).
Comparisons of whole states run on the device (torch views of the engine's
memory)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import ctypes as C

from moonlab_b200 import StateVector, _lib
from moonlab_b200.circuits import config_c2, config_c3

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).resolve().parent / "golden" / "c2_prefix_30q.npz"
TOL = 1e-12


class _View:
    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_view(sv):
    """A torch view of the state's memory once its queued kernels are done
    (they run on the state's own stream, torch reads on its current one)."""
    import torch
    ptr = sv.device_ptr()
    sv.synchronize()
    return torch.as_tensor(_View(ptr, sv.dim, "<c16" if sv.dtype == "c128" else "<c8"), device="cuda")


def max_abs_diff(a, b, chunk=1 << 26):
    m = 0.0
    for off in range(0, a.numel(), chunk):
        m = max(m, float((a[off:off + chunk].to(b.dtype) - b[off:off + chunk]).abs().max()))
    return m


def fidelity(ref, x, chunk=1 << 26):
    import torch
    ip = torch.zeros((), dtype=torch.complex128, device="cuda")
    nx = 0.0
    for off in range(0, ref.numel(), chunk):
        xx = x[off:off + chunk].to(torch.complex128)
        ip += torch.vdot(ref[off:off + chunk], xx)
        nx += float(torch.vdot(xx, xx).real)
    return float(ip.abs() ** 2) / nx


@pytest.mark.skipif(not FIXTURE.exists(), reason="30-qubit reference fixture not generated")
def test_c2_prefix_matches_the_reference(gpu):
    import torch
    f = np.load(FIXTURE)
    n = int(f["n"])
    with StateVector(n) as sv:
        sv.run(f["gates"])
        sv.flush()
        st = sv.flush_stats()
        assert st["dense_blocks"] > 0  # the default c128 path ran dense segments
        a = device_view(sv)
        idx = torch.as_tensor(f["amp_index"], device="cuda")
        got = a[idx].cpu().numpy()
        assert np.abs(got - f["amps"]).max() < TOL
        # <Z_i> as measurement_expectation_z sums it (left to right, FMA):
        # mlb_prob_one_exact reproduces that sum exactly on the engine's
        # amplitudes, so the difference is only the amplitudes' own
        ez = []
        for q in range(n):
            p = C.c_double()
            _lib.check(_lib.load().mlb_prob_one_exact(sv.handle, q, C.byref(p)), "mlb_prob_one_exact")
            ez.append(1.0 - 2.0 * p.value)
        assert np.abs(np.array(ez) - f["ez"]).max() < TOL
        # the one-pass parallel reduction sums 2^30 terms in another order:
        # the reference's serial FP64 sum alone carries ~sqrt(2^30) ulp of rounding
        assert np.abs(sv.expectation_z_all() - f["ez"]).max() < 1e-10
        assert abs(sv.norm_sq() - float(f["norm"])) < 1e-10
        assert np.array_equal(sv.sample(f["uniforms"]), f["outcomes"])


def test_c2_dense_matches_gate_by_gate_at_full_depth(gpu):
    gates, shots = config_c2(30, 40)
    with StateVector(30) as a, StateVector(30) as b:
        a.run(gates)
        b.set_dense(False)
        b.run(gates)
        a.flush()
        b.flush()
        assert a.flush_stats()["dense_blocks"] > 0 and b.flush_stats()["dense_blocks"] == 0
        assert max_abs_diff(device_view(a), device_view(b)) < TOL
        assert abs(a.norm_sq() - 1.0) < 1e-11
        sa = a.sample(shots)
        assert np.array_equal(sa, b.sample(shots))
        with StateVector(30, "c64") as c:
            c.set_exec_mode("fused")
            c.run(gates)
            assert fidelity(device_view(a), device_view(c)) >= 1 - 1e-6


@pytest.mark.parametrize("n,dtype", [(33, "c128"), (34, "c64")])
def test_capacity_limits_keep_the_norm(gpu, n, dtype):
    import torch
    torch.cuda.empty_cache()  # 128 GiB states: no cached torch blocks beside them
    gates = config_c3(n, 20)
    with StateVector(n, dtype) as sv:
        if dtype == "c64":
            sv.set_exec_mode("fused")
        sv.run(gates)
        p1 = sv.probability_one_all()
        norm = sv.norm_sq()
        outs = sv.sample(np.linspace(0.01, 0.99, 64))
    assert abs(norm - 1.0) < (1e-10 if dtype == "c128" else 1e-3)
    assert np.all((p1 >= 0) & (p1 <= norm * (1 + 1e-12)))
    assert outs.max() < (1 << n) and np.all(np.diff(outs.astype(np.float64)) >= 0)  # increasing uniforms


def test_c64_against_c128_at_32_qubits(gpu):
    gates = config_c3(32, 20)
    with StateVector(32) as a, StateVector(32, "c64") as b:
        a.run(gates)
        b.set_exec_mode("fused")
        b.run(gates)
        assert fidelity(device_view(a), device_view(b)) >= 1 - 1e-6
