"""Braket result types on the device (snuqs_b200.result_types through
StateVectorSimulation) against numpy restatements of the observables'
semantics on the oracle state."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import adjoint, circuits
from snuqs_b200 import observables as obs
from snuqs_b200 import result_types as rt
from snuqs_b200.simulation import StateVectorSimulation
from tests.test_observables_cpu import embed

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def _expect(psi, m):
    return float(np.real(np.vdot(psi, m @ psi)))


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-12), ("complex64", 1e-5)])
def test_result_types_against_dense_observables(precision, tol):
    n = 6
    ops = circuits.random_all_gates(n, 120, seed=21)
    ref = oracle.run_ops(ops, n)
    sim = StateVectorSimulation(n, shots=0, precision=precision)
    sim.evolve(ops)
    rng = np.random.default_rng(3)
    a = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    herm = a + a.conj().T
    cases = [
        (obs.PauliX([2]), embed(np.array([[0, 1], [1, 0]], dtype=complex), [2], n)),
        (obs.Hadamard([5]), embed(np.array([[1, 1], [1, -1]]) / np.sqrt(2), [5], n)),
        (obs.Hermitian(herm, [4, 1]), embed(herm, [4, 1], n)),
        (obs.TensorProduct([obs.PauliY([0]), obs.Hermitian(herm, [3, 2])]),
         embed(np.kron(np.array([[0, -1j], [1j, 0]]), herm), [0, 3, 2], n)),
    ]
    for o, m in cases:
        e = rt.Expectation(o).calculate(sim)
        v = rt.Variance(o).calculate(sim)
        want_e = _expect(ref, m)
        want_v = _expect(ref, m @ m) - want_e ** 2
        assert abs(e - want_e) <= tol * max(1, abs(want_e)), o
        assert abs(v - want_v) <= tol * max(1, abs(want_v)), o
    # An untargeted observable: one value per qubit.
    per_q = rt.Expectation(obs.PauliZ()).calculate(sim)
    zz = [_expect(ref, embed(np.diag([1.0, -1.0]).astype(complex), [q], n)) for q in range(n)]
    assert np.allclose(per_q, zz, atol=tol)
    p = rt.Probability([4, 0]).calculate(sim)
    assert np.abs(p - oracle.marginal_probabilities(ref, n, [4, 0])).max() <= tol
    assert np.abs(rt.Probability().calculate(sim) - np.abs(ref) ** 2).max() <= tol
    amps = rt.Amplitude(["000000", "101101", "111111"]).calculate(sim)
    for s, val in amps.items():
        assert abs(val - ref[int(s, 2)]) <= tol
    sv = rt.StateVector().calculate(sim)
    assert np.abs(sv - ref).max() <= tol
    sim.close()


def test_samples_come_from_the_device_sampler():
    n = 12
    ops = circuits.random_all_gates(n, 100, seed=4)
    sim = StateVectorSimulation(n, shots=20000, seed=7)
    sim.evolve(ops)
    s = sim.retrieve_samples()
    u = np.random.default_rng(7).random(20000)
    assert np.array_equal(s.astype(np.uint64), oracle.sample_inverse_cdf(oracle.run_ops(ops, n), u))
    sim.close()


def test_adjoint_gradient_result_type():
    n, p = 8, 2
    edges = circuits.random_regular_graph(n, 3, seed=2)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for layer in range(p):
        ops += [("ZZ", (i, j), (0.0,), (layer,)) for i, j in edges]
        ops += [("RotX", (q,), (0.0,), (p + layer,)) for q in range(n)]
    theta = np.random.default_rng(1).uniform(0, np.pi, 2 * p)
    observable = obs.TensorProduct([obs.PauliZ([0]), obs.PauliZ([1])])
    sim = StateVectorSimulation(n)
    sim.evolve(adjoint.bind(ops, theta))
    res = rt.AdjointGradient(observable, theta, ["g0", "g1", "b0", "b1"]).calculate(sim)
    terms = observable.pauli_terms(n)
    h = 1e-6
    for k, name in enumerate(["g0", "g1", "b0", "b1"]):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        ep = oracle.expectation(oracle.run_ops([op[:3] for op in adjoint.bind(ops, tp)], n), n, terms)
        em = oracle.expectation(oracle.run_ops([op[:3] for op in adjoint.bind(ops, tm)], n), n, terms)
        assert abs(res["gradient"][name] - (ep - em) / (2 * h)) <= 1e-7
    e = oracle.expectation(oracle.run_ops([op[:3] for op in adjoint.bind(ops, theta)], n), n, terms)
    assert abs(res["expectation"] - e) <= 1e-12
    sim.close()
