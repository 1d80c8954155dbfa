"""Observables of the Braket result types, as Pauli sums for the engine.

Mirrors the observable classes of the reference plugin
(src/braket/snuqs/observables.py: Identity :33, Hadamard :102, PauliX :136,
PauliY :170, PauliZ :207, Hermitian :245, TensorProduct :329) -- same names,
targets, measured qubits, eigenvalues and fix_qubit -- but where the
reference multiplies a host copy of the state by the observable's matrix
(`apply`), these reduce every observable to a real-weighted sum of Pauli
strings, `pauli_terms(num_qubits)`, which the device evaluates in one pass
per Pauli flip group (sq_expect_pauli) and squares on the fly for the
variance (sq_variance_pauli).  A k-qubit Hermitian matrix M has the exact
decomposition M = sum_P Tr(P M) / 2^k  P over the 4^k Pauli strings P of its
targets; a tensor product multiplies its factors' decompositions.
"""
from __future__ import annotations

import functools
import itertools
import math
from typing import Optional, Sequence

import numpy as np

_P1 = {
    "I": np.eye(2, dtype=np.complex128),
    "X": np.array([[0, 1], [1, 0]], dtype=np.complex128),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    "Z": np.array([[1, 0], [0, -1]], dtype=np.complex128),
}


def _targets(targets, count: Optional[int] = None) -> Optional[tuple[int, ...]]:
    if targets is None:
        return None
    t = tuple(int(q) for q in targets)
    if count is not None and len(t) != count:
        raise ValueError(f"observable acts on {count} qubit(s), got targets {t}")
    if len(set(t)) != len(t):
        raise ValueError(f"repeated target qubit in {t}")
    return t


class Observable:
    """A Hermitian operator on `measured_qubits` (None: not yet targeted)."""

    num_qubits = 1

    def __init__(self, targets: Optional[Sequence[int]] = None):
        self._measured_qubits = _targets(targets, self.num_qubits)

    @property
    def measured_qubits(self) -> Optional[tuple[int, ...]]:
        return self._measured_qubits

    @property
    def targets(self) -> tuple[int, ...]:
        return self._measured_qubits or ()

    def fix_qubit(self, qubit: int) -> "Observable":
        return type(self)([qubit])

    def local_terms(self) -> list[tuple[float, str]]:
        """Pauli decomposition on the observable's own qubits (string index
        j acts on measured_qubits[j])."""
        raise NotImplementedError

    @property
    def eigenvalues(self) -> np.ndarray:
        raise NotImplementedError

    def pauli_terms(self, num_qubits: int) -> list[tuple[float, str]]:
        """Real-weighted Pauli strings of length num_qubits (character q acts
        on qubit q) whose sum is this observable."""
        if self._measured_qubits is None:
            raise ValueError("observable has no target qubits")
        out = []
        for w, local in self.local_terms():
            s = ["I"] * num_qubits
            for q, ch in zip(self._measured_qubits, local):
                if q >= num_qubits:
                    raise ValueError(f"qubit {q} outside a {num_qubits}-qubit state")
                s[q] = ch
            out.append((w, "".join(s)))
        return out


class Identity(Observable):
    def local_terms(self):
        return [(1.0, "I")]

    @property
    def eigenvalues(self):
        return np.array([1.0, 1.0])


class PauliX(Observable):
    def local_terms(self):
        return [(1.0, "X")]

    @property
    def eigenvalues(self):
        return np.array([1.0, -1.0])


class PauliY(Observable):
    def local_terms(self):
        return [(1.0, "Y")]

    @property
    def eigenvalues(self):
        return np.array([1.0, -1.0])


class PauliZ(Observable):
    def local_terms(self):
        return [(1.0, "Z")]

    @property
    def eigenvalues(self):
        return np.array([1.0, -1.0])


class Hadamard(Observable):
    """(X + Z) / sqrt(2)."""

    def local_terms(self):
        r = 1.0 / math.sqrt(2.0)
        return [(r, "X"), (r, "Z")]

    @property
    def eigenvalues(self):
        return np.array([1.0, -1.0])


class Hermitian(Observable):
    """Any Hermitian matrix on k qubits (row/column index: targets[0] is the
    most significant bit), decomposed over the 4^k Pauli strings."""

    def __init__(self, matrix: np.ndarray, targets: Optional[Sequence[int]] = None):
        m = np.asarray(matrix, dtype=np.complex128)
        if m.ndim != 2 or m.shape[0] != m.shape[1] or m.shape[0] & (m.shape[0] - 1) or m.shape[0] < 2:
            raise ValueError("Hermitian observable needs a 2^k x 2^k matrix")
        if not np.allclose(m, m.conj().T, atol=1e-10):
            raise ValueError("matrix is not Hermitian")
        self._matrix = m
        self.num_qubits = int(m.shape[0]).bit_length() - 1
        super().__init__(targets)

    @property
    def matrix(self) -> np.ndarray:
        return self._matrix

    def fix_qubit(self, qubit: int) -> "Observable":
        if self.num_qubits != 1:
            raise ValueError("only a 1-qubit Hermitian can be fixed to one qubit")
        return Hermitian(self._matrix, [qubit])

    @property
    def eigenvalues(self):
        return np.linalg.eigvalsh(self._matrix)

    def local_terms(self):
        return _hermitian_terms(self._matrix.tobytes(), self.num_qubits)


@functools.lru_cache(maxsize=64)
def _hermitian_terms(mbytes: bytes, k: int) -> list[tuple[float, str]]:
    m = np.frombuffer(mbytes, dtype=np.complex128).reshape(1 << k, 1 << k)
    out = []
    for letters in itertools.product("IXYZ", repeat=k):
        p = functools.reduce(np.kron, [_P1[c] for c in letters])
        c = np.trace(p @ m) / (1 << k)
        if abs(c) > 1e-14:
            out.append((float(c.real), "".join(letters)))
    return out


class TensorProduct(Observable):
    """Product of observables on disjoint qubits (reference :329-418)."""

    def __init__(self, factors: Sequence[Observable]):
        if len(factors) < 2:
            raise ValueError("a tensor product needs at least two factors")
        qs = []
        for f in factors:
            if f.measured_qubits is None:
                raise ValueError("every factor of a tensor product needs targets")
            qs += list(f.measured_qubits)
        self._factors = tuple(factors)
        self.num_qubits = len(qs)
        super().__init__(qs)

    @property
    def factors(self) -> tuple[Observable, ...]:
        return self._factors

    def fix_qubit(self, qubit: int) -> "Observable":
        raise ValueError("a tensor product is always targeted")

    @property
    def eigenvalues(self):
        ev = np.array([1.0])
        for f in self._factors:
            ev = np.kron(ev, f.eigenvalues)
        return ev

    def local_terms(self):
        terms = [(1.0, "")]
        for f in self._factors:
            terms = [(w1 * w2, s1 + s2) for w1, s1 in terms for w2, s2 in f.local_terms()]
        return terms


def matrix_of_terms(terms: Sequence[tuple[float, str]]) -> np.ndarray:
    """Dense matrix of a Pauli sum (string index 0 = most significant bit);
    for checks on small sizes."""
    n = len(terms[0][1])
    out = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    for w, s in terms:
        out += w * functools.reduce(np.kron, [_P1[c] for c in s])
    return out
