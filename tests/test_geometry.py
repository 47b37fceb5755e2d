"""Quantum geometry of the hardware-efficient ansatz (moonlab_b200.geometry)
against the reference's own verbs: moonlab_vqe_qgt, moonlab_vqe_berry_curvature
(src/applications/moonlab_vqe_export.c:53-90) and
vqe_natural_gradient_direction (src/algorithms/vqe_qng.c:270-282).

On the CPU: the identity the engine is built on -- the reference's
derivative state (-i/2) U_after G_i U_upto |hf> equals psi(theta + pi e_i)/2
-- with the oracle running the shifted circuits and the tensors assembled
here as the reference assembles them; and the natural-gradient elimination,
singular systems included.  On the GPU: the engine's batched path
(mlb_hea_geometry)."""
from __future__ import annotations

import numpy as np
import pytest

from moonlab_b200 import geometry as G
from moonlab_b200.circuits import config_c4
from oracle import bindings as B

pytestmark_ref = pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")

PROBLEMS = [(4, 2, 0b0101, 0x61), (5, 3, 0b00011, 0x62), (6, 2, 0, 0x63)]


def problem(n, layers, seed):
    return config_c4(n=n, layers=layers, batch=1, num_terms=8, seed=seed)


def shifted_state_tensors(n, layers, params, hf):
    """(metric, curvature) from psi and psi(theta + pi e_i) / 2 run by the
    oracle, filled as vqe_qng.c:166-232 fills them."""
    rows = G.shifted_parameters(params)
    S = np.stack([B.port_run(n, G.hea_gates(n, layers, r, hf)) for r in rows])
    psi, D = S[0], 0.5 * S[1:]
    ov = D @ psi.conj()
    Q = D.conj() @ D.T - np.outer(ov.conj(), ov)
    P = len(ov)
    g, f = np.zeros((P, P)), np.zeros((P, P))
    iu = np.triu_indices(P)
    g[iu] = Q.real[iu]
    g = g + np.triu(g, 1).T
    iu1 = np.triu_indices(P, 1)
    f[iu1] = -2.0 * Q.imag[iu1]
    f = f - f.T
    return g, f


@pytestmark_ref
@pytest.mark.parametrize("n,layers,hf,seed", PROBLEMS)
def test_shifted_states_give_the_reference_geometry(n, layers, hf, seed):
    prob = problem(n, layers, seed)
    params = prob.params[0]
    ref = B.RefSolver(n, layers, prob.paulis, prob.coeffs, hf_reference=hf)
    try:
        g_ref = ref.qgt(params)
        f_ref = ref.berry_curvature(params)
    finally:
        ref.close()
    g, f = shifted_state_tensors(n, layers, params, hf)
    assert np.abs(g - g_ref).max() < 1e-12
    assert np.abs(f - f_ref).max() < 1e-12
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
        g = ref.qgt(params)
    finally:
        ref.close()
    got = G.natural_gradient_direction(g, grad, 1e-2)
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())


@pytestmark_ref
def test_singular_metric_is_refused_as_the_reference_does():
    # from |00> with every angle 0 the RZ derivative states are phases of psi:
    # their metric rows are exactly zero, and without regularization the
    # reference's elimination meets a zero pivot (returns -1; the verb -3)
    ref = B.RefSolver(2, 1, ["ZI", "IZ"], [1.0, 0.5])
    try:
        params = np.zeros(4)
        g = ref.qgt(params)
        assert not g[1].any() and not g[3].any()
        with pytest.raises(RuntimeError):
            ref.natural_gradient(params, np.ones(4), 0.0)
        want = ref.natural_gradient(params, np.ones(4), 1e-3)
    finally:
        ref.close()
    assert G.natural_gradient_direction(g, np.ones(4), 0.0) is None
    assert np.array_equal(G.natural_gradient_direction(g, np.ones(4), 1e-3), want)


def test_shifted_parameters():
    th = np.array([0.1, -0.2, 0.3])
    S = G.shifted_parameters(th)
    assert S.shape == (4, 3) and np.array_equal(S[0], th)
    assert np.array_equal(S[2], th + np.array([0.0, np.pi, 0.0]))


def test_ansatz_records():
    g = G.hea_gates(3, 1, np.arange(6) * 0.1, hf_reference=0b101, insert=3)
    types = [int(t) for t in g["type"]]
    # X X | RY RZ (q0) RY RZ+Z (q1: parameter 3 is q1's RZ) RY RZ (q2) | CNOT CNOT
    assert types == [1, 1, 8, 9, 8, 9, 3, 8, 9, 10, 10]
    assert [int(c) for c in g["control"][-2:]] == [0, 1] and [int(t) for t in g["target"][-2:]] == [1, 2]
    with pytest.raises(ValueError):
        G.hea_gates(3, 1, np.zeros(5))


@pytest.mark.gpu
@pytestmark_ref
@pytest.mark.parametrize("n,layers,hf,seed", PROBLEMS + [(11, 2, 0b10000000101, 0x64)])
def test_engine_geometry_matches_the_reference(gpu, n, layers, hf, seed):
    prob = problem(n, layers, seed)
    params = prob.params[0]
    ref = B.RefSolver(n, layers, prob.paulis, prob.coeffs, hf_reference=hf)
    try:
        g_ref, f_ref = ref.qgt(params), ref.berry_curvature(params)
    finally:
        ref.close()
    g, f = G.geometry(n, layers, params, hf)
    assert np.abs(g - g_ref).max() < 1e-12
    assert np.abs(f - f_ref).max() < 1e-12
