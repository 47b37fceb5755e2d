"""Scheduler jobs and the "b200" backend plug-in.

CPU: the moonlab_job_to_json reader against text the reference wrote
(golden fixture, and live from the reference library when built here), its
error handling, and registration into the reference's backend registry
(scheduler.c:283-305) without running anything.
GPU: outcomes of mlb_job_run and of moonlab_scheduler_run(job, "b200") are
bit-identical to the reference's "simulator" backend (scheduler.c:194-239)
given the same seed."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from moonlab_b200 import _lib
from moonlab_b200.circuits import GATE_DTYPE, brickwork
from moonlab_b200.scheduler import parse_job_json, register_backend, run_job
from oracle import bindings as B

TWO_Q = (10, 11, 12, 13)  # types whose JSON carries "control" (scheduler.c:521-526)
PARAM = (7, 8, 9)


def same_gates(got, want):
    assert len(got) == len(want)
    assert np.array_equal(got["type"], want["type"])
    assert np.array_equal(got["target"], want["target"])
    two = np.isin(want["type"], TWO_Q)
    assert np.array_equal(got["control"][two], want["control"][two])
    assert np.all(got["control"][~two] == -1)
    par = np.isin(want["type"], PARAM)
    assert np.array_equal(got["theta"][par].view(np.uint64), want["theta"][par].view(np.uint64))


def test_parse_reference_job_json(golden):
    desc, gates = parse_job_json(str(golden["sched_json"]))
    assert desc == {"num_qubits": 10, "num_shots": 1000, "num_workers": int(golden["sched_workers"]),
                    "rng_seed": int(golden["sched_seed"])}
    same_gates(gates, golden["sched_gates"])


def test_parse_is_key_order_free_and_checks_input():
    text = ('{"gates": [{"theta": 0.5, "target": 1, "type": 7}, {"control": 0, "type": 10, "target": 2,'
            ' "extra": [1, {"a": null}]}], "rng_seed": "0x00000000000000ff", "num_qubits": 3,'
            ' "schema": "moonlab/job/v0.7.0", "num_shots": 8}')
    desc, g = parse_job_json(text)
    assert desc == {"num_qubits": 3, "num_shots": 8, "num_workers": 1, "rng_seed": 255}
    assert list(g["type"]) == [7, 10] and g["theta"][0] == 0.5 and g["control"][1] == 0
    lib = _lib.load()
    d, n = _lib.MlbJobDesc(), C.c_size_t()
    for bad in ['', '{', '{"num_qubits": 3}', '{"num_qubits": 3, "gates": [{"type": 1}]}',
                '{"num_qubits": 3, "gates": []} x', '{"num_qubits": "3", "gates": []}',
                '{"num_qubits": 3, "gates": [], "rng_seed": "0xZZ"}']:
        assert lib.mlb_job_parse_json(bad.encode(), C.byref(d), None, 0, C.byref(n)) == -6, bad
    # too small a gate buffer reports the count it needs
    buf = np.zeros(1, dtype=GATE_DTYPE)
    assert lib.mlb_job_parse_json(text.encode(), C.byref(d), buf.ctypes.data_as(C.c_void_p), 1,
                                  C.byref(n)) == -6
    assert n.value == 2


def _ref_job(L, n, gates, shots, workers, seed, backend=None):
    job = L.moonlab_job_create(n)
    for gr in gates:
        par = C.c_double(float(gr["theta"]))
        assert L.moonlab_job_add_gate(job, int(gr["type"]), int(gr["target"]), int(gr["control"]),
                                      C.byref(par) if int(gr["type"]) in PARAM else None) == 0
    L.moonlab_job_set_num_shots(job, shots)
    L.moonlab_job_set_num_workers(job, workers)
    L.moonlab_job_set_rng_seed(job, seed)
    if backend:
        L.moonlab_job_set_backend.argtypes = [C.c_void_p, C.c_char_p]
        assert L.moonlab_job_set_backend(job, backend.encode()) == 0
    return job


@pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")
def test_live_reference_json_round_trip():
    L = B.ref()
    g = brickwork(7, 5, 0xAB)
    g = g[np.isin(g["type"], (7, 8, 9, 10))]
    job = _ref_job(L, 7, g, 77, 3, 0xFEEDF00D)
    buf = C.create_string_buffer(1 << 20)
    assert L.moonlab_job_to_json(job, buf, len(buf)) > 0
    L.moonlab_job_free(job)
    desc, gates = parse_job_json(buf.value.decode())
    assert desc == {"num_qubits": 7, "num_shots": 77, "num_workers": 3, "rng_seed": 0xFEEDF00D}
    same_gates(gates, g)


@pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")
def test_register_into_reference_registry():
    L = B.ref()  # opened RTLD_LOCAL: registration takes its function pointers
    assert register_backend(L) == 0
    L.moonlab_find_backend.argtypes = [C.c_char_p]
    L.moonlab_find_backend.restype = C.c_void_p
    be = L.moonlab_find_backend(b"b200")
    assert be
    name = C.cast(C.c_void_p.from_address(be).value, C.c_char_p).value
    assert name == b"b200"
    assert L.moonlab_find_backend(b"simulator")  # the default stays registered
    # registering again replaces, not duplicates (scheduler.c:293-298)
    assert register_backend(L) == 0


# ---------------------------------------------------------------------------
@pytest.mark.gpu
def test_job_run_matches_reference_simulator_golden(gpu, golden):
    desc, gates = parse_job_json(str(golden["sched_json"]))
    out, workers, _ = run_job(desc["num_qubits"], gates, desc["num_shots"], desc["num_workers"],
                              desc["rng_seed"])
    assert workers == desc["num_workers"]
    assert np.array_equal(out, golden["sched_outcomes"])


@pytest.mark.gpu
def test_job_run_matches_oracle_scheduler(gpu):
    g = brickwork(16, 12, 0x77)
    for shots, workers in ((4096, 8), (5, 9), (1, 1)):
        out, used, _ = run_job(16, g, shots, workers, 0xC0FFEE)
        want = np.empty(shots, dtype=np.uint64)
        sv = B.to_svo(g)
        assert B.port().svo_scheduler_simulator(16, sv, len(sv), shots, workers, 0xC0FFEE,
                                                want.ctypes.data_as(C.POINTER(C.c_uint64))) == 0
        assert used == min(workers, shots)
        assert np.array_equal(out, want)


@pytest.mark.gpu
@pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")
def test_reference_scheduler_runs_b200_backend(gpu):
    L = B.ref()
    assert register_backend(L) == 0
    g = brickwork(12, 10, 0x1D)
    g = g[np.isin(g["type"], (7, 8, 9, 10))]
    results = []
    for backend in ("simulator", "b200"):
        job = _ref_job(L, 12, g, 2000, 3, 0xBADC0DE, backend)
        res = B.JobResults()
        assert L.moonlab_scheduler_run(job, C.byref(res)) == 0
        assert res.total_shots == 2000 and res.num_workers_used == 3 and res.num_qubits == 12
        results.append(np.ctypeslib.as_array(res.outcomes, shape=(2000,)).copy())
        L.moonlab_job_results_free(C.byref(res))
        L.moonlab_job_free(job)
    assert np.array_equal(results[0], results[1])
    # error path: no shots -> MOONLAB_SCHED_BAD_ARG from the scheduler itself
    job = _ref_job(L, 12, g, 0, 1, 1, "b200")
    res = B.JobResults()
    assert L.moonlab_scheduler_run(job, C.byref(res)) == -501
    L.moonlab_job_free(job)
    _lib.load().moonlab_b200_release_backend_state()
