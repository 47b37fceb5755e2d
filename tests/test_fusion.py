"""The single-qubit gate-fusion API of the drop-in (fuse_circuit_*, fuse_append_*,
fuse_compile, fuse_execute; src/optimization/fusion/fusion.h) against the
reference's own fusion.c on the same circuits.

CPU: fuse_compile's statistics and fused record counts, and the append
validation, equal the reference's (both are host code).  GPU: fuse_execute of
the fused circuit on a GPU-backed state and on a host state equals the
reference's fuse_execute of the same circuit to 1e-12 per amplitude."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from moonlab_b200 import _lib
from oracle import bindings as B

pytestmark = pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")

ONE = ["h", "x", "y", "z", "s", "sdg", "t", "tdg"]
ONE_T = ["phase", "rx", "ry", "rz"]
TWO = ["cnot", "cz", "cy", "swap"]
TWO_T = ["cphase", "crx", "cry", "crz"]


class FuseStats(C.Structure):
    _fields_ = [("original_gates", C.c_size_t), ("fused_gates", C.c_size_t), ("merges_applied", C.c_size_t)]


def _bind(lib):
    """fuse_* signatures on a library handle (ours or the reference's)."""
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    lib.fuse_circuit_create.restype = vp
    lib.fuse_circuit_create.argtypes = [C.c_size_t]
    lib.fuse_circuit_free.argtypes = [vp]
    lib.fuse_circuit_free.restype = None
    lib.fuse_circuit_len.restype = C.c_size_t
    lib.fuse_circuit_len.argtypes = [vp]
    lib.fuse_circuit_num_qubits.restype = C.c_size_t
    lib.fuse_circuit_num_qubits.argtypes = [vp]
    lib.fuse_compile.restype = vp
    lib.fuse_compile.argtypes = [vp, C.POINTER(FuseStats)]
    lib.fuse_execute.restype = i
    lib.fuse_execute.argtypes = [vp, vp]
    for k in ONE:
        getattr(lib, f"fuse_append_{k}").argtypes = [vp, i]
    for k in ONE_T:
        getattr(lib, f"fuse_append_{k}").argtypes = [vp, i, d]
    for k in TWO:
        getattr(lib, f"fuse_append_{k}").argtypes = [vp, i, i]
    for k in TWO_T:
        getattr(lib, f"fuse_append_{k}").argtypes = [vp, i, i, d]
    lib.fuse_append_u3.argtypes = [vp, i, d, d, d]
    return lib


def random_program(n, length, seed):
    """A list of (name, args) fuse_append calls: runs of 1-qubit gates broken
    by 2-qubit gates, every kind represented."""
    rng = np.random.default_rng(seed)
    prog = []
    for _ in range(length):
        r = rng.random()
        q = int(rng.integers(n))
        if r < 0.35:
            prog.append((ONE[rng.integers(len(ONE))], (q,)))
        elif r < 0.65:
            prog.append((ONE_T[rng.integers(len(ONE_T))], (q, float(rng.uniform(-7, 7)))))
        elif r < 0.72:
            prog.append(("u3", (q,) + tuple(float(x) for x in rng.uniform(-4, 4, 3))))
        else:
            a, b = (int(x) for x in rng.choice(n, 2, replace=False))
            if rng.random() < 0.5:
                prog.append((TWO[rng.integers(len(TWO))], (a, b)))
            else:
                prog.append((TWO_T[rng.integers(len(TWO_T))], (a, b, float(rng.uniform(-7, 7)))))
    return prog


def build(lib, n, prog):
    c = lib.fuse_circuit_create(n)
    assert c
    for name, args in prog:
        assert getattr(lib, f"fuse_append_{name}")(c, *args) == 0
    return c


def compile_both(n, prog):
    ours, ref = _bind(_lib.load()), _bind(B.ref())
    out = []
    for lib in (ours, ref):
        c = build(lib, n, prog)
        st = FuseStats()
        f = lib.fuse_compile(c, C.byref(st))
        assert f
        out.append((lib, c, f, (st.original_gates, st.fused_gates, st.merges_applied), lib.fuse_circuit_len(f)))
    return out


@pytest.mark.parametrize("n,length,seed", [(3, 40, 1), (6, 200, 2), (10, 500, 3)])
def test_compile_matches_the_reference(n, length, seed):
    (lo, co, fo, so, lo_len), (lr, cr, fr, sr, lr_len) = compile_both(n, random_program(n, length, seed))
    try:
        assert so == sr and lo_len == lr_len
        assert so[0] == length and so[1] < length
    finally:
        for lib, c, f in ((lo, co, fo), (lr, cr, fr)):
            lib.fuse_circuit_free(f)
            lib.fuse_circuit_free(c)


@pytest.mark.parametrize("n,length,seed,fused", [(5, 200, 21, True), (7, 300, 22, False), (8, 400, 23, True)])
def test_lowered_ops_match_the_reference_execute(n, length, seed, fused):
    """fuse_execute's engine ops (mlb_fuse_circuit_ops), replayed in numpy
    with the engine's op semantics, equal the reference's fuse_execute on a
    host state: every record kind, fused or not, mapped right."""
    from test_tile_plan import apply_op
    (lo, co, fo, _, _), (lr, cr, fr, _, _) = compile_both(n, random_program(n, length, seed))
    try:
        lib = _lib.load()
        lib.mlb_fuse_circuit_ops.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t,
                                             C.POINTER(C.c_size_t)]
        src = fo if fused else co
        cnt = C.c_size_t()
        assert lib.mlb_fuse_circuit_ops(src, n, None, 0, C.byref(cnt)) == 0
        ops = (_lib.MlbOp * cnt.value)()
        assert lib.mlb_fuse_circuit_ops(src, n, ops, cnt.value, C.byref(cnt)) == 0
        got = np.zeros(1 << n, dtype=np.complex128)
        got[0] = 1
        for o in ops:
            apply_op(got, n, o)
        want_s = B.RefStateVector(n)
        assert lr.fuse_execute(fr if fused else cr, C.byref(want_s.s)) == 0
        want = want_s.amplitudes()
        want_s.close()
        assert np.abs(got - want).max() < 1e-12
    finally:
        for lib_, c, f in ((lo, co, fo), (lr, cr, fr)):
            lib_.fuse_circuit_free(f)
            lib_.fuse_circuit_free(c)


def test_validation_matches_the_reference():
    for lib in (_bind(_lib.load()), _bind(B.ref())):
        assert not lib.fuse_circuit_create(0) and not lib.fuse_circuit_create(33)
        c = lib.fuse_circuit_create(4)
        assert lib.fuse_append_h(c, 4) == -1 and lib.fuse_append_h(c, -1) == -1
        assert lib.fuse_append_cnot(c, 1, 1) == -1 and lib.fuse_append_cz(c, 0, 4) == -1
        assert lib.fuse_append_rx(c, 3, 0.5) == 0 and lib.fuse_circuit_len(c) == 1
        assert lib.fuse_circuit_num_qubits(c) == 4 and lib.fuse_circuit_len(None) == 0
        assert lib.fuse_execute(None, None) == -2  # QS_ERROR_INVALID_STATE
        lib.fuse_circuit_free(c)
        lib.fuse_circuit_free(None)


@pytest.mark.gpu
@pytest.mark.parametrize("n,length,seed", [(6, 300, 11), (13, 800, 12), (16, 1200, 13)])
def test_execute_matches_the_reference(gpu, n, length, seed):
    prog = random_program(n, length, seed)
    (lo, co, fo, _, _), (lr, cr, fr, _, _) = compile_both(n, prog)
    lib = _lib.load()
    try:
        # reference: fused circuit on its own host state
        want_s = B.RefStateVector(n)
        assert lr.fuse_execute(fr, C.byref(want_s.s)) == 0
        want = want_s.amplitudes()
        want_s.close()
        # ours on a GPU-backed state (quantum_state_create_gpu), read back by sync_to_host
        sp = C.POINTER(_lib.QuantumState)()
        assert lib.quantum_state_create_gpu(n, C.byref(sp)) == 0
        assert lo.fuse_execute(fo, sp) == 0
        assert lib.quantum_state_sync_to_host(sp) == 0
        got = np.ctypeslib.as_array((C.c_double * (2 << n)).from_address(sp.contents.amplitudes)).view(
            np.complex128).copy()
        assert np.abs(got - want).max() < 1e-12
        # ours on a host state: uploaded, run and read back
        amps = np.zeros(1 << n, dtype=np.complex128)
        amps[0] = 1.0
        hs = _lib.QuantumState(num_qubits=n, state_dim=1 << n, amplitudes=amps.ctypes.data)
        assert lo.fuse_execute(fo, C.byref(hs)) == 0
        assert np.abs(amps - want).max() < 1e-12
        # the unfused circuit gives the same state
        amps2 = np.zeros(1 << n, dtype=np.complex128)
        amps2[0] = 1.0
        hs2 = _lib.QuantumState(num_qubits=n, state_dim=1 << n, amplitudes=amps2.ctypes.data)
        assert lo.fuse_execute(co, C.byref(hs2)) == 0
        assert np.abs(amps2 - want).max() < 1e-12
        # a state with fewer qubits than the circuit
        small = _lib.QuantumState(num_qubits=n - 1, state_dim=1 << (n - 1), amplitudes=amps.ctypes.data)
        assert lo.fuse_execute(fo, C.byref(small)) == -5  # QS_ERROR_INVALID_DIMENSION
    finally:
        for L_, c, f in ((lo, co, fo), (lr, cr, fr)):
            L_.fuse_circuit_free(f)
            L_.fuse_circuit_free(c)
