"""Pin the CPU oracle (oracle/sv_oracle.c) to the reference: against the
golden fixtures generated by calling the reference's own library
(tests/golden/gen_golden.py), and live against that library when it was
built here (oracle/_ref/liboracle.so)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import corpus_case
from moonlab_b200.circuits import GATE_DTYPE, SplitMix64, brickwork
from oracle import bindings as B


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_corpus_amplitudes(golden):
    worst = 0.0
    for k in range(len(golden["corpus_n"])):
        n, gates, amps = corpus_case(golden, k)
        worst = max(worst, float(np.abs(B.port_run(n, gates) - amps).max()))
    assert worst < 1e-14, worst


def test_corpus_sampling_is_bit_exact(golden):
    u = golden["sample_uniforms"]
    for k in range(len(golden["corpus_n"])):
        _, _, amps = corpus_case(golden, k)
        assert np.array_equal(B.port_sample(amps, u), golden["corpus_sample"][k])
        assert np.array_equal(B.port_measure_all_indices(amps, u[:64]), golden["corpus_measure_all"][k])


def test_corpus_reductions(golden):
    lib = B.port()
    ez = golden["corpus_ez"]
    off = 0
    for k in range(len(golden["corpus_n"])):
        n, _, amps = corpus_case(golden, k)
        av = np.ascontiguousarray(amps).view(np.float64)
        for q in range(n):
            assert lib.svo_expectation_z(_dp(av), n, q) == ez[off + q]  # same loop, same rounding
        off += n
        assert abs(lib.svo_expectation_x(_dp(av), n, 0) - golden["corpus_ex0"][k]) < 1e-15
        assert abs(lib.svo_expectation_y(_dp(av), n, 0) - golden["corpus_ey0"][k]) < 1e-15
        assert abs(lib.svo_correlation_zz(_dp(av), n, 0, 1) - golden["corpus_zz01"][k]) < 1e-15


def test_brickwork12(golden):
    a = B.port_run(12, golden["bw12_gates"])
    assert np.abs(a - golden["bw12_amps"]).max() < 1e-14
    assert np.abs(B.port_probabilities(a) - golden["bw12_probs"]).max() < 1e-16


def test_qgtl_execute_shots(golden):
    g = golden["bw12_gates"]
    g = g[[t in (7, 8, 9, 10) for t in g["type"]]]
    sv = B.to_svo(g)
    outs = np.empty(1024, dtype=np.uint64)
    probs = np.empty(4096, dtype=np.float64)
    rc = B.port().svo_qgtl_execute(12, sv, len(sv), 1024, int(golden["bw12_qgtl_seed"]),
                                   outs.ctypes.data_as(C.POINTER(C.c_uint64)), _dp(probs))
    assert rc == 0
    assert np.array_equal(outs, golden["bw12_qgtl_outcomes"])
    assert np.abs(probs - golden["bw12_qgtl_probs"]).max() < 1e-16


def test_scheduler_simulator_backend(golden):
    g = golden["sched_gates"]
    sv = B.to_svo(g)
    outs = np.empty(1000, dtype=np.uint64)
    rc = B.port().svo_scheduler_simulator(10, sv, len(sv), 1000, int(golden["sched_workers"]),
                                          int(golden["sched_seed"]),
                                          outs.ctypes.data_as(C.POINTER(C.c_uint64)))
    assert rc == 0
    assert np.array_equal(outs, golden["sched_outcomes"])


@pytest.mark.parametrize("tag", ["vqe4", "vqe6"])
def test_hea_adjoint_gradient(golden, tag):
    n, layers = (int(x) for x in golden[f"{tag}_shape"])
    paulis = [str(p) for p in golden[f"{tag}_paulis"]]
    coeffs = golden[f"{tag}_coeffs"]
    pstr = "".join(paulis).encode()
    for params, want in zip(golden[f"{tag}_params"], golden[f"{tag}_grads"]):
        g = np.empty(2 * n * layers)
        e = C.c_double()
        p = np.ascontiguousarray(params)
        rc = B.port().svo_hea_energy_and_gradient(n, layers, 0, _dp(p), len(paulis), _dp(coeffs),
                                                  pstr, C.byref(e), _dp(g))
        assert rc == 0
        assert np.abs(g - want).max() < 1e-12


@pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")
def test_live_against_reference_library():
    """Random deep circuits over the full named-gate set, random states for
    sampling, and the collapse rules, compared with the reference's library."""
    rng = SplitMix64(0xBEEF)
    L = B.ref()
    for n in (3, 7, 11):
        recs = []
        for _ in range(300):
            t = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 20, 21, 22, 23, 24, 25, 26, 27][
                int(rng.uniform() * 21)]
            a = int(rng.uniform() * n)
            b = (a + 1 + int(rng.uniform() * (n - 1))) % n
            recs.append((t, b, a, 0, 6.283 * rng.uniform() - 3.1))
        g = np.array(recs, dtype=GATE_DTYPE)
        r = B.RefStateVector(n)
        r.run(g)
        ref_amps = r.amplitudes()
        assert np.abs(B.port_run(n, g) - ref_amps).max() < 1e-13
        u = rng.uniforms(500)
        assert np.array_equal(B.port_sample(ref_amps, u), r.sample(u))
        # measurement_single_qubit: outcome and collapsed state
        for q in range(n):
            uu = rng.uniform()
            cl = B.RefState()
            L.quantum_state_clone(C.byref(cl), C.byref(r.s))
            want = L.measurement_single_qubit(C.byref(cl), q, uu)
            got_state = ref_amps.copy()
            got = B.port().svo_measurement_single_qubit(_dp(got_state.view(np.float64)), n, q, uu)
            assert got == want
            ref_post = np.frombuffer((C.c_double * (2 << n)).from_address(cl.amplitudes),
                                     dtype=np.complex128)
            assert np.array_equal(got_state, ref_post)
            L.quantum_state_free(C.byref(cl))
        r.close()


def test_numpy_op_reference_matches_the_oracle():
    """The numpy reference of the random-op GPU tests (tests/ops_np.py) gives
    the oracle's results for every op kind the oracle has a kernel for: 1q and
    2q matrices, multi-controlled X and Z, SWAP, Fredkin, ZZ and the
    controlled rotations (its control masking is the same code for 1q, X and
    SWAP)."""
    from ops_np import np_apply, rand_unitary
    n = 7
    rng = np.random.default_rng(77)
    lib = B.port()

    def gate(a, t, q0, q1=-1, q2=-1, th=0.0):
        g = B.SvoGate(t, q0, q1, q2, th, 0.0, 0.0)
        assert lib.svo_apply_gate(_dp(a.view(np.float64)), n, C.byref(g)) == 0

    def rot(axis, th):
        c, s = np.cos(th / 2), np.sin(th / 2)
        if axis == "x":
            return np.array([[c, -1j * s], [-1j * s, c]])
        if axis == "y":
            return np.array([[c, -s], [s, c]], complex)
        return np.diag([np.exp(-0.5j * th), np.exp(0.5j * th)])

    codes = {"x": 24, "y": 25, "z": 26}  # SVO_CRX, SVO_CRY, SVO_CRZ
    for trial in range(60):
        a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        a /= np.linalg.norm(a)
        q = [int(v) for v in rng.permutation(n)]
        t, t2 = q[0], q[1]
        ctrls = q[2:2 + int(rng.integers(0, 3))]
        cmask = sum(1 << c for c in ctrls)
        got = np.ascontiguousarray(a.copy())
        kind = trial % 7
        if kind == 0:
            m = rand_unitary(rng, 2)
            want = np_apply(a, n, "1q", t, -1, 0, m.reshape(4))
            mm = np.ascontiguousarray(m.reshape(4)).view(np.float64)
            lib.svo_apply_1q_matrix(_dp(got.view(np.float64)), n, t, _dp(mm))
        elif kind == 1:
            axis = "xyz"[trial % 3]
            th = float(rng.uniform(-3, 3))
            want = np_apply(a, n, "1q", t, -1, 1 << q[2], rot(axis, th).reshape(4))
            gate(got, codes[axis], q[2], t, th=th)
        elif kind == 2:
            want = np_apply(a, n, "x", t, -1, cmask, None)
            lib.svo_apply_mcx(_dp(got.view(np.float64)), n, cmask, t)
        elif kind == 3:
            m = rand_unitary(rng, 4)
            want = np_apply(a, n, "2q", t, t2, 0, m.reshape(16))
            mm = np.ascontiguousarray(m.reshape(16)).view(np.float64)
            lib.svo_apply_2q_matrix(_dp(got.view(np.float64)), n, t, t2, _dp(mm))
        elif kind == 4:
            if trial % 2:
                want = np_apply(a, n, "swap", t, t2, 0, None)
                gate(got, 13, t, t2)  # SVO_SWAP
            else:
                want = np_apply(a, n, "swap", t, t2, 1 << q[2], None)
                gate(got, 29, q[2], t, t2)  # SVO_FREDKIN
        elif kind == 5:
            th = float(rng.uniform(0, 6.28))
            want = np_apply(a, n, "zz", t, t2, 0, np.array([np.exp(-0.5j * th), np.exp(0.5j * th)]))
            gate(got, 27, t, t2, th=th)  # SVO_ZZ
        else:
            mask = (1 << t) | cmask
            want = np_apply(a, n, "phase", 0, -1, mask, np.array([-1.0]))
            lib.svo_apply_mcz(_dp(got.view(np.float64)), n, mask)
        assert np.abs(got - want).max() < 1e-13, (trial, kind)
