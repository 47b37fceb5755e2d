"""GPU parity: the CUDA engine (through its C ABI) against the reference's
results -- committed golden fixtures made by the reference library, and
the CPU oracle (oracle/sv_oracle.c, pinned to the reference by
test_oracle_pin.py) on the same seeded inputs.

Tolerances: complex128 amplitudes 1e-12 per amplitude (the contract of the
plain path); probabilities, exact sequential sums and sampled outcomes
bit-exact; parallel FP64 reductions 1e-12; complex64 fidelity >= 1 - 1e-6.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import corpus_case
from moonlab_b200 import StateVector, _lib
from moonlab_b200.circuits import GATE_DTYPE, SplitMix64, brickwork, config_c1, qaoa_circuit
from oracle import bindings as B
from ops_np import np_apply, rand_unitary

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def gpu_run(n, gates, mode="tiled", dtype="c128"):
    sv = StateVector(n, dtype)
    sv.set_exec_mode(mode)
    sv.run(gates)
    return sv


def cdf_of(a):
    """The reference's CDF: sequential sum of fl(cabs(a)^2) (measurement.c:569-575)."""
    h = np.abs(a.astype(np.complex128))  # hypot, as cabs
    return np.cumsum(h * h)


# ---------------------------------------------------------------------------
# corpus (the reference's own 75-circuit oracle corpus)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("mode", ["tiled", "eager"])
def test_corpus_amplitudes(gpu, golden, mode):
    worst = 0.0
    for k in range(len(golden["corpus_n"])):
        n, gates, amps = corpus_case(golden, k)
        with gpu_run(n, gates, mode) as sv:
            worst = max(worst, float(np.abs(sv.amplitudes() - amps).max()))
    assert worst < TOL, worst


def test_corpus_sampling_bit_exact(gpu, golden):
    u = golden["sample_uniforms"]
    for k in range(len(golden["corpus_n"])):
        n, _, amps = corpus_case(golden, k)
        with StateVector(n) as sv:
            sv.set_amplitudes(amps)
            assert np.array_equal(sv.sample(u, _lib.MLB_SAMPLE_CDF_GE), golden["corpus_sample"][k])
            assert np.array_equal(sv.sample(u[:64], _lib.MLB_SAMPLE_CUM_GT),
                                  golden["corpus_measure_all"][k])


def test_corpus_expectations(gpu, golden):
    ez = golden["corpus_ez"]
    off = 0
    for k in range(len(golden["corpus_n"])):
        n, _, amps = corpus_case(golden, k)
        with StateVector(n) as sv:
            sv.set_amplitudes(amps)
            for q in range(n):
                p = C.c_double()
                _lib.check(_lib.load().mlb_prob_one_exact(sv.handle, q, C.byref(p)), "prob_one_exact")
                assert 1.0 - 2.0 * p.value == ez[off + q]  # bit-identical to measurement_expectation_z
            assert np.abs(sv.expectation_z_all() - ez[off:off + n]).max() < TOL
            assert abs(sv.expectation_pauli(1, 0) - golden["corpus_ex0"][k]) < TOL
            assert abs(sv.expectation_pauli(1, 1) - golden["corpus_ey0"][k]) < TOL
            assert abs(sv.correlation_zz(0, 1) - golden["corpus_zz01"][k]) < TOL
            off += n


# ---------------------------------------------------------------------------
# the 20-qubit brickwork workload
# ---------------------------------------------------------------------------
def test_brickwork20_end_to_end(gpu):
    gates, shots = config_c1()
    want = B.port_run(20, gates)
    with gpu_run(20, gates) as sv:
        got = sv.amplitudes()
        assert np.abs(got - want).max() < TOL
        assert np.array_equal(sv.probabilities(0), B.port_probabilities(got, 0))
        assert np.array_equal(sv.probabilities(1), B.port_probabilities(got, 1))
        assert np.abs(sv.expectation_z_all() - np.array(
            [B.port().svo_expectation_z(_dp(want.view(np.float64)), 20, q) for q in range(20)])).max() < TOL
        s = sv.sample(shots)
        assert np.array_equal(s, B.port_sample(got, shots))
        assert np.array_equal(s, B.port_sample(want, shots))
        assert abs(sv.norm_sq() - 1.0) < 1e-12


def test_brickwork_eager_equals_tiled(gpu):
    g = brickwork(16, 12, 99, zz_every=3)
    with gpu_run(16, g, "tiled") as a, gpu_run(16, g, "eager") as b:
        assert np.abs(a.amplitudes() - b.amplitudes()).max() < TOL
    assert np.abs(B.port_run(16, g) - gpu_run(16, g).amplitudes()).max() < TOL


# ---------------------------------------------------------------------------
# all-zero tiles: after a reset, passes run only over tiles that may be nonzero
# ---------------------------------------------------------------------------
def test_zero_tiles_skipped_after_reset(gpu):
    n = 22
    g1 = brickwork(n, 6, 11, zz_every=2)
    g2 = brickwork(n, 5, 12, zz_every=3)
    full = 2 * 16 * (1 << n)
    with StateVector(n) as sv, StateVector(n) as other:
        # from |0...0>: the first passes touch a few tiles only
        sv.run(g1)
        a1 = sv.amplitudes()
        st = sv.flush_stats()
        assert np.abs(a1 - B.port_run(n, g1)).max() < TOL
        assert st["bytes_moved"] < st["passes"] * full
        assert st["dense_amps"] < st["dense_blocks"] << n
        # a second circuit on the now dense state: every tile
        sv.run(g2)
        a12 = sv.amplitudes()
        st = sv.flush_stats()
        assert np.abs(a12 - B.port_run_from(n, g2, a1)).max() < TOL
        assert st["bytes_moved"] == st["passes"] * full
        # collapse to a basis state, then more gates: only its index is nonzero
        k = sv.measure_all(0.61)
        basis = np.zeros(1 << n, complex)
        basis[k] = 1
        assert np.array_equal(sv.amplitudes(), basis)
        sv.run(g1)
        assert np.abs(sv.amplitudes() - B.port_run_from(n, g1, basis)).max() < TOL
        assert sv.flush_stats()["bytes_moved"] < sv.flush_stats()["passes"] * full
        # a copy of a fresh state keeps its zero tiles; uploaded amplitudes do not
        sv.reset()
        other.copy_from(sv)
        other.run(g2)
        assert np.abs(other.amplitudes() - B.port_run(n, g2)).max() < TOL
        assert other.flush_stats()["bytes_moved"] < other.flush_stats()["passes"] * full
        other.set_amplitudes(a1)
        other.run(g2)
        assert np.abs(other.amplitudes() - a12).max() < TOL
        assert other.flush_stats()["bytes_moved"] == other.flush_stats()["passes"] * full
        # after the device pointer is handed out, every pass runs over every tile
        other.device_ptr()
        other.reset()
        other.run(g1)
        assert np.abs(other.amplitudes() - a1).max() < TOL
        assert other.flush_stats()["bytes_moved"] == other.flush_stats()["passes"] * full
    # the fused complex64 path skips the same tiles
    with StateVector(n, "c64") as f:
        f.run(g1)
        got = f.amplitudes().astype(np.complex128)  # flushes
        st = f.flush_stats()
        assert abs(np.vdot(a1, got)) ** 2 / np.vdot(got, got).real >= 1 - 1e-6
        assert 0 < st["bytes_moved"] < st["passes"] * (full // 2)
        f.run(g2)
        got = f.amplitudes().astype(np.complex128)
        st = f.flush_stats()
        assert abs(np.vdot(a12, got)) ** 2 / np.vdot(got, got).real >= 1 - 1e-6
        assert st["bytes_moved"] == st["passes"] * (full // 2)


# ---------------------------------------------------------------------------
# QAOA: CNOT . RZ . CNOT lifted to one parity-phase op per edge
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n,mode,dense", [(12, "tiled", True), (16, "tiled", True), (16, "tiled", False),
                                          (16, "eager", True), (20, "tiled", True)])
def test_qaoa_parity_phases(gpu, n, mode, dense):
    g = qaoa_circuit(n, 3, 0x9A0A ^ n)
    want = B.port_run(n, g)
    with StateVector(n, "c128") as sv:
        sv.set_exec_mode(mode)
        sv.set_dense(dense)
        sv.run(g)
        got = sv.amplitudes()
        st = sv.flush_stats()
    assert np.abs(got - want).max() < TOL
    if mode == "tiled":
        assert st["ops"] < len(g)  # the sandwiches were lifted


def test_qaoa_fused_c64(gpu):
    n = 16
    g = qaoa_circuit(n, 3, 0x9A0A ^ n)
    want = B.port_run(n, g)
    with StateVector(n, "c64") as sv:
        sv.set_exec_mode("fused")
        sv.run(g)
        got = sv.amplitudes().astype(np.complex128)
    fid = abs(np.vdot(want, got)) ** 2 / np.vdot(got, got).real
    assert fid >= 1 - 1e-6


# ---------------------------------------------------------------------------
# every op kind, controls and targets inside and outside a tile
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n,mode,dtype", [(9, "tiled", "c128"), (13, "tiled", "c128"), (15, "tiled", "c128"),
                                          (15, "eager", "c128"), (17, "tiled", "c128"), (22, "tiled", "c128"),
                                          (15, "tiled", "c64")])
def test_random_ops_all_kinds(gpu, n, mode, dtype):
    rng = np.random.default_rng(1234 + n)
    a = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n))
    a /= np.linalg.norm(a)
    want = a.copy()
    with StateVector(n, dtype) as sv:
        sv.set_exec_mode(mode)
        sv.set_amplitudes(a)
        for _ in range(160):
            kind = ["1q", "x", "2q", "swap", "zz", "phase", "c1q"][rng.integers(7)]
            qs = rng.permutation(n)
            t, t2 = int(qs[0]), int(qs[1])
            nc = int(rng.integers(0, 3))
            ctrls = [int(c) for c in qs[2:2 + nc]]
            cmask = sum(1 << c for c in ctrls)
            if kind in ("1q", "c1q"):
                m = rand_unitary(rng, 2)
                if kind == "c1q":
                    sv.apply_controlled_1q(ctrls, t, m)
                else:
                    sv.apply_1q(t, m)
                    cmask = 0
                want = np_apply(want, n, "1q", t, -1, cmask, m.reshape(4))
            elif kind == "x":
                sv.mcx(ctrls, t)
                want = np_apply(want, n, "x", t, -1, cmask, None)
            elif kind == "2q":
                m = rand_unitary(rng, 4)
                sv.apply_2q(t, t2, m)
                want = np_apply(want, n, "2q", t, t2, 0, m.reshape(16))
            elif kind == "swap":
                sv.cswap(ctrls, t, t2)
                want = np_apply(want, n, "swap", t, t2, cmask, None)
            elif kind == "zz":
                th = float(rng.uniform(0, 6.28))
                sv.zz(t, t2, th)
                want = np_apply(want, n, "zz", t, t2, 0,
                                np.array([np.exp(-0.5j * th), np.exp(0.5j * th)]))
            else:
                qq = [t] + ctrls
                sv.mcz(qq)
                want = np_apply(want, n, "phase", 0, -1, sum(1 << q for q in qq), np.array([-1.0]))
        got = sv.amplitudes()
        st = sv.flush_stats()
    if dtype == "c128" and mode == "tiled" and n >= 13:
        assert st["dense_blocks"] > 0  # some segments ran on the FP64 tensor cores
    tol = TOL if dtype == "c128" else 2e-5
    assert np.abs(got - want).max() < tol


@pytest.mark.parametrize("n,depth", [(16, 12), (20, 8)])
def test_dense_segments_match_gate_by_gate(gpu, n, depth):
    """complex128 tile passes with their segments as dense matrices on the
    FP64 tensor cores (the default) and gate by gate agree with the oracle
    to 1e-12 per amplitude; brickwork with ZZ layers and extra controlled
    gates on arbitrary pairs, so segments carry conditioning qubits."""
    g = list(brickwork(n, depth, 0xD5 + n, zz_every=3))
    rng = np.random.default_rng(n)
    for _ in range(20):  # CNOT / CY / SWAP / controlled rotation on random pairs
        a, b = rng.choice(n, 2, replace=False)
        g.insert(int(rng.integers(len(g))), (int(rng.choice([10, 11, 13, 23])), int(b), int(a), 0,
                                             float(rng.uniform(0, 6.28))))
    g = np.array(g, dtype=GATE_DTYPE)
    want = B.port_run(n, g)
    for dense in (True, False):
        with StateVector(n, "c128") as sv:
            sv.set_dense(dense)
            sv.run(g)
            got = sv.amplitudes()
            st = sv.flush_stats()
        assert (st["dense_blocks"] > 0) == dense
        assert np.abs(got - want).max() < TOL, dense


def test_c64_fidelity_on_brickwork20(gpu):
    gates, _ = config_c1()
    with gpu_run(20, gates) as ref128, gpu_run(20, gates, dtype="c64") as s64:
        a = ref128.amplitudes()
        b = s64.amplitudes().astype(np.complex128)
    fid = abs(np.vdot(a, b)) ** 2
    assert fid >= 1.0 - 1e-6, fid
    assert np.abs(a - b).max() < 1e-5


# ---------------------------------------------------------------------------
# sampling and collapse: bit-exact semantics on adversarial states
# ---------------------------------------------------------------------------
def _states(n):
    rng = np.random.default_rng(n)
    d = 1 << n
    zero = np.zeros(d, complex)
    zero[0] = 1
    basis = np.zeros(d, complex)
    basis[d // 3] = 1
    uniform = np.full(d, 1 / np.sqrt(d), complex)
    rnd = rng.standard_normal(d) + 1j * rng.standard_normal(d)
    rnd /= np.linalg.norm(rnd)
    keep = rng.random(d) < 0.05
    keep[rng.integers(0, d, 3)] = True  # never empty
    sparse = np.where(keep, rnd, 0)
    sparse /= np.linalg.norm(sparse)
    tiny = rnd * np.exp(-rng.uniform(0, 300, d))  # probabilities down to ~1e-260
    tiny[d // 2] = 1.0
    tiny /= np.linalg.norm(tiny)
    # exact ties: the running sum stays in [0.5, 1) (grid 2^-53) and every
    # other element adds exactly half a grid step (|2^-27|^2 = 2^-54), so the
    # sum's rounding depends on its parity; the rest fill the sum towards 1
    ties = np.zeros(d, complex)
    ties[0] = 0.5 + 0.5j
    ties[1::2] = 2.0 ** -27
    rest = rnd[2::2] / np.linalg.norm(rnd[2::2]) * np.sqrt(0.49)
    ties[2::2] = rest
    return dict(zero=zero, basis=basis, uniform=uniform, random=rnd, sparse=sparse, tiny=tiny, ties=ties)


@pytest.mark.parametrize("n", [5, 13, 22])
def test_sampling_bit_exact_adversarial(gpu, n):
    rng = np.random.default_rng(7 * n)
    for name, a in _states(n).items():
        cdf = cdf_of(a)
        # uniforms exactly on CDF values (the >= / > boundary), next to them, and random
        picks = cdf[rng.integers(0, a.size, 200)]
        u = np.concatenate([picks, np.nextafter(picks, 0), np.nextafter(picks, 1),
                            rng.random(300), [0.0, 1.0 - 2 ** -53, cdf[-1]]])
        u = u[(u >= 0) & (u < 1)]
        with StateVector(n) as sv:
            sv.set_amplitudes(a)
            ge = sv.sample(u, _lib.MLB_SAMPLE_CDF_GE)
            gt = sv.sample(u, _lib.MLB_SAMPLE_CUM_GT)
        assert np.array_equal(ge, B.port_sample(a, u)), name
        assert np.array_equal(gt, B.port_measure_all_indices(a, u)), name


def _large_states(n):
    """States for the chunk-scan path at 2^(n-12) chunks (several 4096-chunk
    scans): leading runs of all-zero chunks longer than a scan, probabilities
    spread over ~1000 binades, and a dense random state.  Made one at a time."""
    d = 1 << n
    rng = np.random.default_rng(1000 + n)
    basis = np.zeros(d, complex)
    basis[d - d // 3] = 1
    yield "basis", basis
    del basis
    half = np.zeros(d, complex)
    half[d // 2:] = rng.standard_normal(d // 2) + 1j * rng.standard_normal(d // 2)
    half /= np.linalg.norm(half)
    yield "zero_then_random", half
    del half
    rnd = rng.standard_normal(d) + 1j * rng.standard_normal(d)
    rnd /= np.linalg.norm(rnd)
    yield "random", rnd
    rnd *= np.exp(-rng.uniform(0, 300, d))
    rnd[d // 5] = 1.0
    rnd /= np.linalg.norm(rnd)
    yield "tiny", rnd


def test_sampling_bit_exact_many_scan_batches(gpu):
    n = 26
    rng = np.random.default_rng(26)
    for name, a in _large_states(n):
        cdf = cdf_of(a)
        picks = cdf[rng.integers(0, a.size, 100)]
        u = np.concatenate([picks, np.nextafter(picks, 0), np.nextafter(picks, 1), rng.random(200)])
        u = u[(u >= 0) & (u < 1)]
        del cdf
        with StateVector(n) as sv:
            sv.set_amplitudes(a)
            ge = sv.sample(u, _lib.MLB_SAMPLE_CDF_GE)
            u_gt = u[::40]  # the oracle walks the whole state once per uniform here
            gt = sv.sample(u_gt, _lib.MLB_SAMPLE_CUM_GT)
            av = np.ascontiguousarray(a).view(np.float64)
            for q in (0, n - 1):
                p = C.c_double()
                _lib.check(_lib.load().mlb_prob_one_exact(sv.handle, q, C.byref(p)), "prob_one_exact")
                assert p.value == B.port().svo_probability_one(_dp(av), n, q), (name, q)
        assert np.array_equal(ge, B.port_sample(a, u)), name
        assert np.array_equal(gt, B.port_measure_all_indices(a, u_gt)), name


@pytest.mark.parametrize("n", [6, 14, 21])
def test_exact_sequential_sums(gpu, n):
    for name, a in _states(n).items():
        av = np.ascontiguousarray(a).view(np.float64)
        with StateVector(n) as sv:
            sv.set_amplitudes(a)
            for q in sorted({0, n // 2, n - 1}):
                p = C.c_double()
                _lib.check(_lib.load().mlb_prob_one_exact(sv.handle, q, C.byref(p)), "prob_one_exact")
                assert p.value == B.port().svo_probability_one(_dp(av), n, q), (name, q)


@pytest.mark.parametrize("n", [4, 12, 18])
def test_measurement_collapse_bit_exact(gpu, n):
    rng = np.random.default_rng(100 + n)
    for name, a in _states(n).items():
        for q in sorted({0, n // 2, n - 1}):
            u = float(rng.random())
            # measurement_single_qubit
            want = np.ascontiguousarray(a.copy())
            r_want = B.port().svo_measurement_single_qubit(_dp(want.view(np.float64)), n, q, u)
            with StateVector(n) as sv:
                sv.set_amplitudes(a)
                r = sv.measure_qubit(q, u)
                got = sv.amplitudes()
            assert r == r_want, (name, q)
            assert np.array_equal(got, want), (name, q)
            # quantum_measure
            want = np.ascontiguousarray(a.copy())
            pw = C.c_double()
            r_want = B.port().svo_quantum_measure(_dp(want.view(np.float64)), n, q, u, C.byref(pw))
            with StateVector(n) as sv:
                sv.set_amplitudes(a)
                r, p = sv.quantum_measure(q, u)
                got = sv.amplitudes()
            if r_want >= 0:
                assert (r, p) == (r_want, pw.value), (name, q)
                assert np.array_equal(got, want), (name, q)


def test_measure_all_collapses(gpu):
    a = _states(10)["random"]
    u = 0.37
    idx = int(B.port_measure_all_indices(a, [u])[0])
    with StateVector(10) as sv:
        sv.set_amplitudes(a)
        assert sv.measure_all(u) == idx
        post = sv.amplitudes()
    want = np.zeros_like(a)
    want[idx] = 1
    assert np.array_equal(post, want)


# ---------------------------------------------------------------------------
# the drop-in boundary, called the way the reference calls it
# ---------------------------------------------------------------------------
def test_dropin_routes_and_sync(gpu):
    lib = _lib.load()
    n = 13
    qs = C.POINTER(_lib.QuantumState)()
    assert lib.quantum_state_create_gpu(n, C.byref(qs)) == 0
    st = qs.contents
    assert st.gpu_backend == 1 and st.num_qubits == n and st.state_dim == 1 << n
    rng = SplitMix64(5)
    recs = []
    for k in range(120):
        t = int(rng.uniform() * n)
        c = (t + 1 + int(rng.uniform() * (n - 1))) % n
        recs.append([(7, t, -1, 0, rng.uniform() * 6), (10, c, t, 0, 0.0), (4, t, -1, 0, 0.0),
                     (1, t, -1, 0, 0.0), (12, t, c, 0, 0.0), (24, t, c, 0, rng.uniform())][k % 6])
    g = np.array(recs, dtype=GATE_DTYPE)
    from moonlab_b200 import gates_to_ops
    for rec, op in zip(g, gates_to_ops(g, n)):
        t, c = int(rec["target"]), int(rec["control"])
        if rec["type"] == 10:
            assert lib.qsim_gpu_route_cnot(qs, c, t) == 0
        elif rec["type"] == 4:
            assert lib.qsim_gpu_route_hadamard(qs, t) == 0
        elif rec["type"] == 1:
            assert lib.qsim_gpu_route_pauli_x(qs, t) == 0
        elif rec["type"] == 12:
            assert lib.qsim_gpu_route_mcz(qs, (1 << t) | (1 << c)) == 0
        elif rec["type"] == 24:  # controlled RX through the 4x4 route (gates.c:776-799)
            m = np.zeros(32)
            m[0] = m[20] = 1.0
            m[10], m[11], m[14], m[15] = op.m[0], op.m[1], op.m[2], op.m[3]
            m[26], m[27], m[30], m[31] = op.m[4], op.m[5], op.m[6], op.m[7]
            assert lib.qsim_gpu_route_apply_2q_matrix(qs, c, t, _dp(m)) == 0
        else:
            m = np.array(op.m[:8])
            assert lib.qsim_gpu_route_apply_1q_matrix(qs, t, _dp(m)) == 0
    assert lib.quantum_state_sync_to_host(qs) == 0
    host = np.ctypeslib.as_array(C.cast(st.amplitudes, C.POINTER(C.c_double)), shape=(2 << n,)).view(np.complex128)
    want = B.port_run(n, g)
    assert np.abs(host - want).max() < TOL
    # moonlab_cuda_* surface on the same engine state
    eng = C.c_void_p(st.gpu_state)
    nrm, pz = C.c_double(), C.c_double()
    assert lib.moonlab_cuda_norm(eng, C.byref(nrm)) == 0 and abs(nrm.value - 1) < TOL
    assert lib.moonlab_cuda_prob_z(eng, 3, C.byref(pz)) == 0
    assert abs(pz.value - B.port().svo_probability_one(_dp(want.view(np.float64)), n, 3)) < TOL
    assert lib.moonlab_cuda_state_n_qubits(eng) == n and lib.moonlab_cuda_state_dim(eng) == 1 << n
    # sync_from_host round trip
    host[:] = 0
    host[5] = 1
    assert lib.quantum_state_sync_from_host(qs) == 0
    assert lib.moonlab_cuda_prob_z(eng, 0, C.byref(pz)) == 0 and pz.value == 1.0
    assert lib.qsim_gpu_route_cnot(qs, 0, 99) == -1            # invalid qubit -> -1
    assert lib.moonlab_cuda_apply_cnot(eng, 2, 2) == -4         # MOONLAB_CUDA_ERR_INVALID_QUBIT
    lib.moonlab_cuda_state_free(eng)
    assert lib.moonlab_cuda_runtime_probe_discrete() == 1


@pytest.mark.skipif(not B.REF_DROPIN_LIB.exists(), reason="reference core not built here")
def test_reference_core_routes_to_engine(gpu):
    """The reference's own gates.c / measurement.c (built without their CPU
    routing stubs) resolve qsim_gpu_route_* and quantum_state_create_gpu to
    libmoonlab_b200.so, exactly as they would link state_gpu.cu."""
    import os
    _lib.load()  # RTLD_GLOBAL first
    core = C.CDLL(str(B.REF_DROPIN_LIB), mode=os.RTLD_GLOBAL)
    # A program calling quantum_state_create_gpu resolves it in the global
    # scope, where the engine's strong definition (loaded first) precedes the
    # reference's weak stub (state.c:645-651); dlsym on the core's own handle
    # would return the stub instead.
    glob = C.CDLL(None)
    sp = C.POINTER(_lib.QuantumState)
    glob.quantum_state_create_gpu.argtypes = [C.c_size_t, C.POINTER(sp)]
    for name in ("gate_rx", "gate_ry", "gate_rz"):
        getattr(core, name).argtypes = [sp, C.c_int, C.c_double]
    core.gate_cnot.argtypes = [sp, C.c_int, C.c_int]
    core.gate_cz.argtypes = [sp, C.c_int, C.c_int]
    core.gate_hadamard.argtypes = [sp, C.c_int]
    core.measurement_probability_one.argtypes = [sp, C.c_int]
    core.measurement_probability_one.restype = C.c_double
    core.quantum_state_destroy.argtypes = [sp]
    n = 12
    qs = sp()
    assert glob.quantum_state_create_gpu(n, C.byref(qs)) == 0
    assert qs.contents.gpu_backend == 1
    g = brickwork(n, 6, 31)
    for rec in g:
        t, c, th = int(rec["target"]), int(rec["control"]), float(rec["theta"])
        rc = {7: lambda: core.gate_rx(qs, t, th), 8: lambda: core.gate_ry(qs, t, th),
              9: lambda: core.gate_rz(qs, t, th), 10: lambda: core.gate_cnot(qs, c, t)}[int(rec["type"])]()
        assert rc == 0
    assert core.gate_hadamard(qs, 3) == 0 and core.gate_cz(qs, 1, 5) == 0
    g2 = np.concatenate([g, np.array([(4, 3, -1, 0, 0.0), (12, 5, 1, 0, 0.0)], dtype=GATE_DTYPE)])
    want = B.port_run(n, g2)
    p = core.measurement_probability_one(qs, 4)  # pulls through quantum_state_sync_to_host
    assert p == B.port().svo_probability_one(_dp(want.view(np.float64)), n, 4) or abs(
        p - B.port().svo_probability_one(_dp(want.view(np.float64)), n, 4)) < TOL
    host = np.ctypeslib.as_array(C.cast(qs.contents.amplitudes, C.POINTER(C.c_double)),
                                 shape=(2 << n,)).view(np.complex128)
    assert np.abs(host - want).max() < TOL
    core.quantum_state_destroy(qs)


def test_plan_cache_replays_repeated_shapes(gpu):
    """A repeated circuit shape (same gates and qubits, new angles) reuses the
    cached plan and replays its launches as a graph; amplitudes are
    bit-identical to an uncached state's.  A new shape misses; the least
    recently used plan is evicted at capacity."""
    n = 16
    shapes = [brickwork(n, 8, s, zz_every=3) for s in (1, 2, 3)]  # same shape, new angles
    other = brickwork(n, 5, 9)  # different depth: a new shape
    with StateVector(n) as cached, StateVector(n) as plain:
        cached.set_plan_cache(2)
        hits = []
        for g in shapes + [other, shapes[0]]:
            for sv in (cached, plain):
                sv.reset()
                sv.run(g)
                sv.flush()
            hits.append(cached.flush_stats()["plan_cache_hit"])
            assert np.array_equal(cached.amplitudes(), plain.amplitudes())
        assert hits == [0, 1, 1, 0, 1]
        cached.set_plan_cache(1)  # shrinking drops the cache
        cached.reset()
        cached.run(other)
        cached.flush()
        assert cached.flush_stats()["plan_cache_hit"] == 0
        a = cached.amplitudes()
        want = B.port_run(n, other)
        assert np.abs(a - want).max() < TOL


def test_fp64_tensor_probe(gpu):
    # the roofline denominator of the dense complex128 segments: a B200 runs
    # mma.sync f64 at tens of TFLOP/s (nominal FP64 tensor rate about 40)
    v = C.c_double()
    assert gpu.mlb_fp64_tensor_peak(0, C.byref(v)) == 0
    assert 15.0 < v.value < 60.0
