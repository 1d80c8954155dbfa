"""Observables as Pauli sums (no GPU): every observable's decomposition
rebuilds its matrix exactly, tensor products multiply, untargeted observables
fix to each qubit, and the oracle's sampling walk is an inverse CDF."""
import functools

import numpy as np
import pytest

import oracle
from snuqs_b200 import observables as obs
from snuqs_b200 import result_types as rt

H = np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2)
MATS = {obs.PauliX: np.array([[0, 1], [1, 0]]), obs.PauliY: np.array([[0, -1j], [1j, 0]]),
        obs.PauliZ: np.diag([1, -1]), obs.Hadamard: H, obs.Identity: np.eye(2)}


def embed(m, targets, n):
    """Dense matrix of m acting on `targets` of n qubits (qubit 0 = MSB)."""
    k = len(targets)
    full = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    rest = [q for q in range(n) if q not in targets]
    for i in range(1 << n):
        bits = [(i >> (n - 1 - q)) & 1 for q in range(n)]
        r = int("".join(str(bits[q]) for q in targets), 2) if k else 0
        for c in range(1 << k):
            j_bits = list(bits)
            for t, q in enumerate(targets):
                j_bits[q] = (c >> (k - 1 - t)) & 1
            j = int("".join(map(str, j_bits)), 2)
            full[i, j] += m[r, c]
    del rest
    return full


@pytest.mark.parametrize("cls", list(MATS))
def test_single_qubit_observables(cls):
    n = 3
    for q in range(n):
        o = cls([q])
        got = obs.matrix_of_terms(o.pauli_terms(n))
        assert np.allclose(got, embed(np.asarray(MATS[cls], dtype=np.complex128), [q], n), atol=1e-14)
        assert np.allclose(sorted(o.eigenvalues), sorted(np.linalg.eigvalsh(MATS[cls])))


def test_hermitian_and_tensor_product():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
    m = a + a.conj().T
    n = 4
    h = obs.Hermitian(m, [3, 1])
    assert np.allclose(obs.matrix_of_terms(h.pauli_terms(n)), embed(m, [3, 1], n), atol=1e-12)
    t = obs.TensorProduct([obs.PauliX([0]), obs.Hermitian(m, [2, 3])])
    want = embed(np.kron(MATS[obs.PauliX], m), [0, 2, 3], n)
    assert np.allclose(obs.matrix_of_terms(t.pauli_terms(n)), want, atol=1e-12)
    assert sorted(t.eigenvalues) == pytest.approx(sorted(np.linalg.eigvalsh(np.kron(MATS[obs.PauliX], m))))
    with pytest.raises(ValueError):
        obs.Hermitian(a, [0, 1])  # not Hermitian
    with pytest.raises(ValueError):
        obs.TensorProduct([obs.PauliZ([0]), obs.PauliZ([0])])


def test_untargeted_observable_fixes_to_each_qubit():
    z = obs.PauliZ()
    assert z.measured_qubits is None
    assert [z.fix_qubit(q).pauli_terms(3) for q in range(3)] == [
        [(1.0, "ZII")], [(1.0, "IZI")], [(1.0, "IIZ")]]


def test_braket_ir_observables():
    o = rt.from_braket_observable(["x", "z"], [2, 0])
    assert o.pauli_terms(3) == [(1.0, "ZIX")]
    m = [[[1, 0], [0, 0]], [[0, 0], [-1, 0]]]
    o = rt.from_braket_observable([m], [1])
    assert np.allclose(obs.matrix_of_terms(o.pauli_terms(2)), embed(np.diag([1, -1]), [1], 2))
    with pytest.raises(ValueError):
        rt.from_braket_observable(["x", "z"], [2, 0, 1])


def test_amplitude_validates_states():
    with pytest.raises(ValueError):
        rt.Amplitude([])


def test_oracle_sampling_walk_is_an_inverse_cdf():
    rng = np.random.default_rng(0)
    for n in (1, 5, 13):
        psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        u = rng.random(20000)
        idx = oracle.sample_inverse_cdf(psi, u).astype(np.int64)
        p = np.abs(psi) ** 2
        c = np.cumsum(p)
        j = np.searchsorted(c, u * c[-1], side="right")
        assert (idx == j).mean() > 0.999
        assert np.all(p[idx] > 0)
    # zero-probability amplitudes are never drawn
    psi = np.zeros(64, dtype=np.complex128)
    psi[[3, 40]] = [0.6, 0.8]
    idx = oracle.sample_inverse_cdf(psi, np.linspace(0, 1, 1000, endpoint=False))
    assert set(idx.tolist()) == {3, 40}
