"""Adjoint gradients on the GPU: against central finite differences of the
oracle's energy, and against the parameter-shift rule on the same engine
(1e-10 for complex128, 1e-4 for complex64)."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import adjoint, capi, circuits
from tests.test_adjoint_cpu import energy as oracle_energy
from tests.test_adjoint_cpu import fd_grad, random_param_circuit

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def qaoa(n, p, seed):
    edges = circuits.random_regular_graph(n, 3, seed=seed)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for l in range(p):
        ops += [("ZZ", (i, j), (0.0,), (l,)) for i, j in edges]
        ops += [("RotX", (q,), (0.0,), (p + l,)) for q in range(n)]
    return ops, circuits.maxcut_hamiltonian(n, edges)


@pytest.mark.parametrize("n,seed", [(5, 0), (9, 1), (12, 2), (14, 3)])
def test_adjoint_vs_finite_differences(n, seed):
    nparams = 6
    ops = random_param_circuit(n, 40, nparams, seed)
    theta = np.random.default_rng(seed + 100).uniform(-3, 3, nparams)
    terms = circuits.random_pauli_hamiltonian(n, 12, seed=seed)
    ws = adjoint.Workspace(n)
    e, g = adjoint.adjoint_gradient(ws, ops, theta, terms, nparams)
    ws.close()
    assert abs(e - oracle_energy(n, ops, theta, terms)) < 1e-11
    assert np.abs(g - fd_grad(n, ops, theta, terms)).max() < 1e-7


@pytest.mark.parametrize("dtype,tol", [(capi.SQ_C128, 1e-10), (capi.SQ_C64, 1e-4)])
def test_adjoint_vs_parameter_shift_qaoa(dtype, tol):
    n, p = 16, 3
    ops, terms = qaoa(n, p, seed=7)
    theta = np.random.default_rng(7).uniform(0, np.pi, 2 * p)
    ws = adjoint.Workspace(n, dtype)
    e, g = adjoint.adjoint_gradient(ws, ops, theta, terms, 2 * p)
    ref = capi.State(n, capi.SQ_C128)
    gs = adjoint.parameter_shift_gradient(ref, ops, theta, terms, 2 * p)
    e_ref = adjoint.energy(ref, ops, theta, terms)
    ref.close()
    ws.close()
    assert abs(e - e_ref) <= tol * max(1.0, abs(e_ref))
    assert np.abs(g - gs).max() <= tol * max(1.0, np.abs(gs).max())


def test_adjoint_general_gates_complex64():
    n, nparams = 13, 5
    ops = random_param_circuit(n, 40, nparams, 9)
    theta = np.random.default_rng(9).uniform(-3, 3, nparams)
    terms = circuits.random_pauli_hamiltonian(n, 10, seed=9)
    ws = adjoint.Workspace(n, capi.SQ_C64)
    e, g = adjoint.adjoint_gradient(ws, ops, theta, terms, nparams)
    ws.close()
    assert abs(e - oracle_energy(n, ops, theta, terms)) < 1e-4
    assert np.abs(g - fd_grad(n, ops, theta, terms)).max() < 1e-4


def test_torch_autograd_function():
    import torch

    n, p = 10, 2
    ops, terms = qaoa(n, p, seed=3)
    ws = adjoint.Workspace(n)
    theta = torch.tensor([0.3, 0.5, 0.7, 0.2], dtype=torch.float64, requires_grad=True)
    e = adjoint.AdjointExpectation.apply(theta, ws, ops, terms)
    e.backward()
    want = fd_grad(n, ops, theta.detach().numpy(), terms)
    ws.close()
    assert np.abs(theta.grad.numpy() - want).max() < 1e-7


def test_adjoint_rejects_bad_input():
    ws = adjoint.Workspace(6)
    with pytest.raises(capi.SqError):
        # parameter index 3 but only 1 parameter: rejected by the C ABI
        adjoint.adjoint_gradient(ws, [("RotX", (0,), (0.1,), (3,))], [0.0] * 4, [(1.0, "ZIIIII")], 1)
    ws.close()


def test_repeated_gradients_on_one_workspace_reuse_plans():
    """Gradients of one circuit at three parameter sets on the same workspace
    (the forward and reverse plans are re-emitted from their recipes after the
    first), each against the parameter-shift rule; 20 qubits, JIT sweeps."""
    n, p = 20, 2
    ops, terms = qaoa(n, p, seed=4)
    ws = adjoint.Workspace(n)
    ref = capi.State(n, capi.SQ_C128)
    rng = np.random.default_rng(4)
    for _ in range(3):
        theta = rng.uniform(0, np.pi, 2 * p)
        e, g = adjoint.adjoint_gradient(ws, ops, theta, terms, 2 * p)
        gs = adjoint.parameter_shift_gradient(ref, ops, theta, terms, 2 * p)
        assert abs(e - adjoint.energy(ref, ops, theta, terms)) <= 1e-10
        assert np.abs(g - gs).max() <= 1e-10 * max(1.0, np.abs(gs).max())
    ref.close()
    ws.close()
