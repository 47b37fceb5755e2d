"""mlb_prob_one_all_noalloc through the C ABI: the probs_z reduction on
caller-owned device buffers with the library's fixed per-device scratch
array.  Checked against mlb_prob_one_all / mlb_norm_sq on the same states
(parallel FP64 reductions: 1e-12), on consecutive calls that reuse the
scratch with different sizes, plus its argument checks.  Collected last, so
it also runs after every other test has used the device."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from moonlab_b200 import StateVector, _lib
from moonlab_b200.circuits import brickwork

pytestmark = pytest.mark.gpu

TOL = 1e-12


def expected(sv):
    return np.append(sv.probability_one_all(), sv.norm_sq())


def noalloc(lib, sv, out, stream):
    dtype = _lib.MLB_C128 if sv.dtype == "c128" else _lib.MLB_C64
    rc = lib.mlb_prob_one_all_noalloc(C.c_void_p(sv.device_ptr()), dtype, sv.n,
                                      C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert rc == 0, lib.mlb_last_error().decode()


def test_noalloc_matches_prob_one_all(gpu):
    import torch
    lib = gpu
    a = StateVector(22, "c128")
    a.run(brickwork(22, 6, seed=0x5EED))
    b = StateVector(16, "c64")
    rng = np.random.default_rng(7)
    amps = (rng.standard_normal(1 << 16) + 1j * rng.standard_normal(1 << 16)).astype(np.complex64)
    b.set_amplitudes(amps * 0.01)  # norm far from 1
    want_a, want_b = expected(a), expected(b)

    out_a = torch.full((23,), float("nan"), dtype=torch.float64, device="cuda")
    out_b = torch.full((17,), float("nan"), dtype=torch.float64, device="cuda")
    # 1st call: on the state's own stream
    noalloc(lib, a, out_a, a.stream())
    a.synchronize()
    got_a1 = out_a.cpu().numpy()
    # 2nd call, right after, on the default stream with a smaller state
    noalloc(lib, b, out_b, 0)
    torch.cuda.synchronize()
    got_b = out_b.cpu().numpy()
    # 3rd: back to the large state over the scratch the small one left behind
    out_a.fill_(float("nan"))
    noalloc(lib, a, out_a, 0)
    torch.cuda.synchronize()
    got_a2 = out_a.cpu().numpy()

    assert np.abs(got_a1 - want_a).max() < TOL
    assert np.abs(got_b - want_b).max() < TOL
    assert np.abs(got_a2 - want_a).max() < TOL
    a.close()
    b.close()


def test_noalloc_rejects_bad_arguments(gpu):
    import torch
    lib = gpu
    out = torch.zeros(32, dtype=torch.float64, device="cuda")
    amp = torch.zeros(2 * 16, dtype=torch.float64, device="cuda")
    ap, op = C.c_void_p(amp.data_ptr()), C.c_void_p(out.data_ptr())
    f = lib.mlb_prob_one_all_noalloc
    assert f(ap, _lib.MLB_C128, 31, op, None) == -5      # above the scratch limit
    assert f(ap, _lib.MLB_C128, 0, op, None) == -5
    assert "1..30" in lib.mlb_last_error().decode()
    assert f(None, _lib.MLB_C128, 4, op, None) == -6
    assert f(ap, 7, 4, op, None) == -6
    host = np.zeros(32)
    assert f(C.c_void_p(host.ctypes.data), _lib.MLB_C128, 4, op, None) == -6  # host memory
    assert f(ap, _lib.MLB_C128, 4, C.c_void_p(host.ctypes.data), None) == -6
    assert f(C.c_void_p(amp.data_ptr() + 8), _lib.MLB_C128, 3, op, None) == -6  # misaligned
    # a good call still works after the rejections
    amp[0] = 1.0
    assert f(ap, _lib.MLB_C128, 4, op, None) == 0
    torch.cuda.synchronize()
    assert out[:5].cpu().tolist() == [0.0, 0.0, 0.0, 0.0, 1.0]
