"""The VQE verbs of the stable ABI on the device, against the reference's
own symbols on the same solver (both resolved from their libraries):

* moonlab_vqe_qgt, moonlab_vqe_berry_curvature, moonlab_vqe_natural_gradient
  (src/applications/moonlab_vqe_export.c:53-100) for the hardware-efficient
  ansatz: psi and the P derivative states as one batch through the forward
  passes, the Gram matrix from the engine's FP64 kernel (mlb_hea_geometry);
* moonlab_vqe_gradient for the UCCSD and symmetry-preserving ansaetze: the
  reference's exact four-term parameter-shift rule (vqe.c:2072-2140) with
  every shifted energy run on the device.

Tolerances: metric and curvature 1e-12 (entries of order 0.1-1, FP64 sums of
2^n terms in a different order); parameter-shift gradients 1e-10 (each a
difference of energies computed in FP64 in a different order); the natural
gradient 1e-9 relative (a P x P solve amplifies the metric's rounding by its
condition number)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from moonlab_b200 import _lib
from moonlab_b200.circuits import config_c4
from oracle import bindings as B

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ours(fn, solver, params, P):
    p = np.ascontiguousarray(params, dtype=np.float64)
    out = np.empty((P, P), dtype=np.float64)
    assert fn(solver, _dp(p), _dp(out), P) == 0
    return out


@pytest.mark.parametrize("n,layers,hf,seed", [(4, 2, 0b0101, 0x71), (7, 3, 0b0010011, 0x72), (10, 2, 0, 0x73)])
def test_geometry_verbs_match_the_reference(gpu, n, layers, hf, seed):
    lib = _lib.load()
    prob = config_c4(n=n, layers=layers, batch=2, num_terms=12, seed=seed)
    s = B.RefSolver(n, layers, prob.paulis, prob.coeffs, hf_reference=hf)
    try:
        P = s.P
        for params in prob.params:
            g_ref, f_ref = s.qgt(params), s.berry_curvature(params)
            g, f = ours(lib.moonlab_vqe_qgt, s.solver, params, P), ours(lib.moonlab_vqe_berry_curvature, s.solver,
                                                                        params, P)
            assert np.abs(g - g_ref).max() < 1e-12
            assert np.abs(f - f_ref).max() < 1e-12
            assert np.array_equal(g, g.T) and np.array_equal(f, -f.T) and not np.diag(f).any()
            grad = s.gradient(params)
            want = s.natural_gradient(params, grad, 1e-2)
            got = np.empty(P)
            pp, gg = np.ascontiguousarray(params), np.ascontiguousarray(grad)
            assert lib.moonlab_vqe_natural_gradient(s.solver, _dp(pp), _dp(gg), C.c_double(1e-2), _dp(got), P) == 0
            assert np.abs(got - want).max() <= 1e-9 * max(1.0, np.abs(want).max())
        # argument checks of moonlab_vqe_export.c:60-65
        out = np.empty((P, P))
        pp = np.ascontiguousarray(prob.params[0])
        assert lib.moonlab_vqe_qgt(None, _dp(pp), _dp(out), P) == -1
        assert lib.moonlab_vqe_qgt(s.solver, _dp(pp), None, P) == -1
        assert lib.moonlab_vqe_berry_curvature(s.solver, _dp(pp), _dp(out), P + 1) == -2
    finally:
        s.close()


def test_singular_metric_is_refused_as_the_reference_does(gpu):
    # from |00> with every angle 0 the RZ derivative states are phases of psi:
    # their metric rows are exactly zero, and without regularization both
    # eliminations meet a zero pivot (the verb returns -3)
    lib = _lib.load()
    n, layers = 2, 1
    s = B.RefSolver(n, layers, ["ZI", "IZ"], [1.0, 0.5])
    try:
        P = s.P
        params = np.zeros(P)
        grad = np.ones(P)
        got = np.empty(P)
        rc_ours = lib.moonlab_vqe_natural_gradient(s.solver, _dp(params), _dp(grad), C.c_double(0.0), _dp(got), P)
        rc_ref = s.lib.moonlab_vqe_natural_gradient(s.solver, _dp(params), _dp(grad), C.c_double(0.0), _dp(got), P)
        assert rc_ref == -3 and rc_ours == -3
    finally:
        s.close()


def test_engine_batch_matches_the_shifted_state_composition(gpu):
    # mlb_hea_geometry (batched shifted states + Gram kernel) against the
    # same tensors assembled from oracle-run shifted states on the CPU, on a
    # register wide enough for several tile passes and Gram tile pairs
    from moonlab_b200.vqe import HEAProblem
    from test_geometry import shifted_state_tensors
    n, layers, hf = 13, 2, 0b1000000000101
    prob = config_c4(n=n, layers=layers, batch=1, num_terms=10, seed=0x74)
    hp = HEAProblem(n, layers, prob.coeffs, paulis=prob.paulis, hf_reference=hf)
    try:
        g, f = hp.geometry(prob.params[0])
    finally:
        hp.close()
    g_cpu, f_cpu = shifted_state_tensors(n, layers, prob.params[0], hf)
    assert np.abs(g - g_cpu).max() < 1e-12
    assert np.abs(f - f_cpu).max() < 1e-12


@pytest.mark.parametrize("kind,n,arg,seed", [("uccsd", 4, (2,), 0x81), ("uccsd", 6, (2,), 0x82),
                                             ("symmetry", 6, (3, 2), 0x83)])
def test_parameter_shift_gradient_matches_the_reference(gpu, kind, n, arg, seed):
    lib = _lib.load()
    prob = config_c4(n=n, layers=1, batch=1, num_terms=3 * n, seed=seed)
    occ = arg[0]
    hf = (1 << occ) - 1 if kind == "uccsd" else ((1 << occ) - 1) << (n - occ)
    s = B.RefSolver(n, 1, prob.paulis, prob.coeffs, hf_reference=hf, ansatz=(kind,) + arg)
    try:
        P = s.P
        rng = np.random.default_rng(seed)
        for _ in range(2):
            params = rng.uniform(-np.pi, np.pi, P)
            want = s.gradient(params)
            got = np.empty(P)
            assert lib.moonlab_vqe_gradient(s.solver, _dp(params), _dp(got), P) == 0
            assert np.abs(got - want).max() < 1e-10
            assert np.abs(want).max() > 1e-3
    finally:
        s.close()
