"""GPU parity of the batched adjoint VQE gradient (hardware-efficient ansatz)
against the reference's moonlab_vqe_gradient (golden fixtures and, where
built, live through the drop-in entry), the CPU oracle's per-term adjoint
restatement, and central finite differences of the engine's own energies.
Tolerances: complex128 gradients 1e-11 absolute vs the reference / oracle;
finite differences (h = 1e-6) within 2e-7; complex64 within 1e-4 relative."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from moonlab_b200 import _lib
from moonlab_b200.circuits import SplitMix64, config_c4
from moonlab_b200.vqe import HEAProblem, pauli_masks
from oracle import bindings as B

pytestmark = pytest.mark.gpu


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def port_energy_grad(n, layers, hf, paulis, coeffs, params):
    g = np.empty(2 * n * layers)
    e = C.c_double()
    p = np.ascontiguousarray(params, dtype=np.float64)
    c = np.ascontiguousarray(coeffs, dtype=np.float64)
    rc = B.port().svo_hea_energy_and_gradient(n, layers, hf, _dp(p), len(paulis), _dp(c),
                                              "".join(paulis).encode(), C.byref(e), _dp(g))
    assert rc == 0
    return e.value, g


def random_problem(n, layers, terms, seed):
    rng = SplitMix64(seed)
    paulis, coeffs = [], []
    for _ in range(terms):
        s = ["I"] * n
        for _ in range(1 + int(rng.uniform() * min(3, n))):
            s[int(rng.uniform() * n)] = "IXYZ"[1 + int(rng.uniform() * 3)]
        paulis.append("".join(s))
        coeffs.append(2 * rng.uniform() - 1)
    params = np.array([[(2 * rng.uniform() - 1) * np.pi for _ in range(2 * n * layers)] for _ in range(3)])
    hf = int(rng.uniform() * (1 << n))
    return paulis, np.array(coeffs), params, hf


@pytest.mark.parametrize("tag", ["vqe4", "vqe6"])
def test_gradients_match_reference_golden(gpu, golden, tag):
    n, layers = (int(x) for x in golden[f"{tag}_shape"])
    paulis = [str(p) for p in golden[f"{tag}_paulis"]]
    prob = HEAProblem(n, layers, golden[f"{tag}_coeffs"], paulis=paulis)
    E, G = prob.evaluate(golden[f"{tag}_params"])
    assert np.abs(G - golden[f"{tag}_grads"]).max() < 1e-11
    for k, p in enumerate(golden[f"{tag}_params"]):
        e_port, _ = port_energy_grad(n, layers, 0, paulis, golden[f"{tag}_coeffs"], p)
        assert abs(E[k] - e_port) < 1e-12


@pytest.mark.parametrize("n,layers,terms", [(2, 2, 5), (3, 1, 6), (7, 3, 20), (12, 2, 30), (14, 1, 40)])
def test_gradients_match_oracle(gpu, n, layers, terms):
    paulis, coeffs, params, hf = random_problem(n, layers, terms, 1000 + n)
    prob = HEAProblem(n, layers, coeffs, paulis=paulis, hf_reference=hf)
    E, G = prob.evaluate(params)
    for k in range(len(params)):
        e_ref, g_ref = port_energy_grad(n, layers, hf, paulis, coeffs, params[k])
        assert abs(E[k] - e_ref) < 1e-11
        assert np.abs(G[k] - g_ref).max() < 1e-11


def test_gradient_vs_finite_differences_20q(gpu):
    prob_def = config_c4(n=20, layers=8, batch=2, num_terms=80, seed=0xC4)
    prob = HEAProblem(20, 8, prob_def.coeffs, xmasks=prob_def.xmasks, zmasks=prob_def.zmasks)
    p0 = prob_def.params[:1]
    _, G = prob.evaluate(p0)
    h = 1e-6
    rng = np.random.default_rng(3)
    idx = rng.choice(prob.num_parameters, 6, replace=False)
    shifted = []
    for i in idx:
        for sgn in (1, -1):
            q = p0[0].copy()
            q[i] += sgn * h
            shifted.append(q)
    E, _ = prob.evaluate(np.array(shifted), want_grad=False)
    fd = (E[0::2] - E[1::2]) / (2 * h)
    scale = max(1.0, np.abs(G).max())
    assert np.abs(fd - G[0][idx]).max() < 2e-7 * scale


def test_complex64_gradients(gpu):
    paulis, coeffs, params, hf = random_problem(12, 3, 24, 77)
    g128 = HEAProblem(12, 3, coeffs, paulis=paulis, hf_reference=hf).evaluate(params)[1]
    g64 = HEAProblem(12, 3, coeffs, paulis=paulis, hf_reference=hf, dtype="c64").evaluate(params)[1]
    assert np.abs(g64 - g128).max() < 1e-4 * max(1.0, np.abs(g128).max())


@pytest.mark.parametrize("n,layers,batch,hf_bits", [(13, 2, 3, 0), (16, 4, 6, 0b101), (18, 3, 8, 0)])
def test_complex64_forward_on_the_tensor_cores(gpu, n, layers, batch, hf_bits):
    """The complex64 forward sweep on the tensor cores (fused <= 5-qubit
    blocks, operand images built per vector on the device) gives the
    energies and gradients of the CUDA-core forward and of complex128 to
    1e-4 relative; batches that are not a power of two, several checkpoint
    segments and an hf reference included."""
    paulis, coeffs, _, _ = random_problem(n, layers, 3 * n, 500 + n)
    rng = np.random.default_rng(n)
    params = rng.uniform(-np.pi, np.pi, (batch, 2 * n * layers))
    p128 = HEAProblem(n, layers, coeffs, paulis=paulis, hf_reference=hf_bits)
    E128, G128 = p128.evaluate(params)
    with pytest.raises(_lib.MlbError):
        p128.set_fused_forward("on")  # complex128 has no fused forward
    p64 = HEAProblem(n, layers, coeffs, paulis=paulis, hf_reference=hf_bits, dtype="c64")
    p64.set_checkpointing("always")
    E_f, G_f = p64.evaluate(params)
    assert p64.last_eval_stats()["fused_forward"]
    p64.set_fused_forward("off")
    E_c, G_c = p64.evaluate(params)
    assert not p64.last_eval_stats()["fused_forward"]
    scale = max(1.0, np.abs(G128).max())
    for E, G in ((E_f, G_f), (E_c, G_c)):
        assert np.abs(E - E128).max() < 1e-4 * max(1.0, np.abs(E128).max())
        assert np.abs(G - G128).max() < 1e-4 * scale
    assert np.abs(G_f - G_c).max() < 1e-4 * scale


def test_sub_batches_under_a_memory_budget(gpu):
    paulis, coeffs, params, hf = random_problem(13, 2, 16, 5)
    prob = HEAProblem(13, 2, coeffs, paulis=paulis, hf_reference=hf)
    E1, G1 = prob.evaluate(params)
    prob.set_memory_budget(2 * 16 << 13)  # room for one (psi, lambda) pair
    E2, G2 = prob.evaluate(params)
    assert np.array_equal(E1, E2) and np.array_equal(G1, G2)


def test_torch_autograd_function(gpu):
    import torch
    from moonlab_b200.vqe import AdjointEnergy
    paulis, coeffs, params, hf = random_problem(10, 2, 12, 9)
    prob = HEAProblem(10, 2, coeffs, paulis=paulis, hf_reference=hf)
    x = torch.tensor(params, dtype=torch.float64, device="cuda", requires_grad=True)
    w = torch.tensor([0.5, -2.0, 1.5], dtype=torch.float64, device="cuda")
    E = AdjointEnergy.apply(x, prob)
    (E * w).sum().backward()
    E_np, G_np = prob.evaluate(params)
    assert np.allclose(E.detach().cpu().numpy(), E_np, atol=1e-13, rtol=0)
    assert np.allclose(x.grad.cpu().numpy(), w.cpu().numpy()[:, None] * G_np, atol=1e-12, rtol=0)


@pytest.mark.skipif(not B.have_ref(), reason="reference library not built here")
def test_dropin_moonlab_vqe_gradient_on_reference_solver(gpu):
    lib = _lib.load()
    n, layers = 6, 3
    paulis, coeffs, params, _ = random_problem(n, layers, 18, 42)
    hf = 0b100101
    s = B.RefSolver(n, layers, paulis, coeffs, hf_reference=hf)
    P = s.P
    for p in params:
        want = s.gradient(p)
        got = np.empty(P)
        pp = np.ascontiguousarray(p)
        assert lib.moonlab_vqe_gradient(s.solver, _dp(pp), _dp(got), P) == 0
        assert np.abs(got - want).max() < 1e-11
    # batched entry
    pp = np.ascontiguousarray(params)
    got = np.empty_like(pp)
    assert lib.moonlab_b200_vqe_gradient_batch(s.solver, len(pp), _dp(pp), _dp(got), P) == 0
    assert np.abs(got[1] - s.gradient(params[1])).max() < 1e-11
    # error codes of moonlab_vqe_export.c:31-37
    g = np.empty(P)
    assert lib.moonlab_vqe_gradient(None, _dp(pp), _dp(g), P) == -1
    assert lib.moonlab_vqe_gradient(s.solver, _dp(pp), _dp(g), P - 1) == -2
    s.close()


def test_checkpointed_backward_sweep(gpu):
    """Checkpoints every ceil(sqrt(L)) layers give the same gradients (the
    restored psi equals the uncomputed one to rounding), and the memory
    policy drops them before splitting the batch."""
    paulis, coeffs, params, hf = random_problem(12, 9, 24, 31)
    prob = HEAProblem(12, 9, coeffs, paulis=paulis, hf_reference=hf)
    prob.set_checkpointing("always")
    E1, G1 = prob.evaluate(params)
    st = prob.last_eval_stats()
    assert st["checkpoints"] and st["segment_layers"] == 3 and st["sub_batches"] == 1
    prob.set_checkpointing("never")
    E2, G2 = prob.evaluate(params)
    assert not prob.last_eval_stats()["checkpoints"]
    assert np.array_equal(E1, E2)
    assert np.abs(G1 - G2).max() < 1e-12
    for k in range(len(params)):
        _, g_ref = port_energy_grad(12, 9, hf, paulis, coeffs, params[k])
        assert np.abs(G1[k] - g_ref).max() < 1e-11
    # auto: a budget for psi + lambda of all 3 vectors but not their 2 checkpoints each
    state = 16 << 12
    prob.set_checkpointing("auto")
    prob.set_memory_budget(3 * 2 * state + state)
    _, G3 = prob.evaluate(params)
    st = prob.last_eval_stats()
    assert not st["checkpoints"] and st["sub_batches"] == 1
    prob.set_memory_budget(3 * 4 * state)
    _, G4 = prob.evaluate(params)
    assert prob.last_eval_stats()["checkpoints"]
    prob.set_memory_budget(2 * state)  # one vector at a time, no room for checkpoints
    _, G5 = prob.evaluate(params)
    st = prob.last_eval_stats()
    assert not st["checkpoints"] and st["sub_batches"] == 3
    for G in (G3, G4, G5):
        assert np.abs(G - G1).max() < 1e-12
