"""Quantum geometry of the hardware-efficient ansatz (moonlab_b200.geometry)
against the reference's own verbs: moonlab_vqe_qgt, moonlab_vqe_berry_curvature
(src/applications/moonlab_vqe_export.c:53-90) and
vqe_natural_gradient_direction (src/algorithms/vqe_qng.c:270-282).  On the
CPU the oracle runs the derivative circuits; on the GPU the engine does."""
from __future__ import annotations

import numpy as np
import pytest

from moonlab_b200 import geometry as G
from moonlab_b200.circuits import config_c4
from oracle import bindings as B

pytestmark_ref = pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")

PROBLEMS = [(4, 2, 0b0101, 0x61), (5, 3, 0b00011, 0x62), (6, 2, 0, 0x63)]


def oracle_runner(n):
    import torch
    return lambda gates: torch.from_numpy(B.port_run(n, gates))


def problem(n, layers, seed):
    return config_c4(n=n, layers=layers, batch=1, num_terms=8, seed=seed)


@pytestmark_ref
@pytest.mark.parametrize("n,layers,hf,seed", PROBLEMS)
def test_metric_and_curvature_match_the_reference(n, layers, hf, seed):
    prob = problem(n, layers, seed)
    params = prob.params[0]
    ref = B.RefSolver(n, layers, prob.paulis, prob.coeffs, hf_reference=hf)
    try:
        g_ref = ref.qgt(params)
        f_ref = ref.berry_curvature(params)
    finally:
        ref.close()
    run = oracle_runner(n)
    g = G.metric(n, layers, params, run, hf)
    f = G.berry_curvature(n, layers, params, run, hf)
    assert np.abs(g - g_ref).max() < 1e-12
    assert np.abs(f - f_ref).max() < 1e-12
    assert np.array_equal(g, g.T) and np.array_equal(f, -f.T)
    assert np.abs(f).max() > 1e-3  # the RZ layers make the state complex: F is not zero


@pytestmark_ref
def test_natural_gradient_direction_matches_the_reference():
    n, layers, hf, seed = PROBLEMS[0]
    prob = problem(n, layers, seed)
    params = prob.params[0]
    ref = B.RefSolver(n, layers, prob.paulis, prob.coeffs, hf_reference=hf)
    try:
        grad = ref.gradient(params)
        want = ref.natural_gradient_direction(params, grad, 1e-2)
    finally:
        ref.close()
    g = G.metric(n, layers, params, oracle_runner(n), hf)
    got = G.natural_gradient_direction(g, grad, 1e-2)
    assert np.abs(got - want).max() <= 1e-9 * max(1.0, np.abs(want).max())


def test_ansatz_records():
    g = G.hea_gates(3, 1, np.arange(6) * 0.1, hf_reference=0b101, insert=3)
    types = [int(t) for t in g["type"]]
    # X X | RY RZ (q0) RY RZ+Z (q1: parameter 3 is q1's RZ) RY RZ (q2) | CNOT CNOT
    assert types == [1, 1, 8, 9, 8, 9, 3, 8, 9, 10, 10]
    assert [int(c) for c in g["control"][-2:]] == [0, 1] and [int(t) for t in g["target"][-2:]] == [1, 2]
    with pytest.raises(ValueError):
        G.hea_gates(3, 1, np.zeros(5))


@pytest.mark.gpu
def test_engine_runner_matches_the_oracle(gpu):
    n, layers, hf = 8, 2, 0b1001
    prob = problem(n, layers, 0x64)
    params = prob.params[0]
    run = G.EngineRunner(n)
    try:
        g_dev = G.metric(n, layers, params, run, hf)
        f_dev = G.berry_curvature(n, layers, params, run, hf)
    finally:
        run.close()
    run_cpu = oracle_runner(n)
    assert np.abs(g_dev - G.metric(n, layers, params, run_cpu, hf)).max() < 1e-12
    assert np.abs(f_dev - G.berry_curvature(n, layers, params, run_cpu, hf)).max() < 1e-12
