"""Noise channels (Kraus operators) of the Braket noise instructions.

The reference plugin defines these channels (src/braket/snuqs/
noise_operations.py:30-384) but its simulator refuses every noise pragma
(src/braket/snuqs/simulator.py:650-659): nothing simulates them.  Here each
channel gives its Kraus operators, and snuqs_b200.density_matrix applies them
on the device as one dense superoperator each.

Definitions (Braket's): with the Paulis I, X, Y, Z,
* BitFlip(p): sqrt(1-p) I, sqrt(p) X;  PhaseFlip(p): sqrt(1-p) I, sqrt(p) Z;
* PauliChannel(px, py, pz): sqrt(1-px-py-pz) I, sqrt(px) X, sqrt(py) Y, sqrt(pz) Z;
* Depolarizing(p): sqrt(1-p) I and sqrt(p/3) each of X, Y, Z;
* TwoQubitDepolarizing(p): sqrt(1-p) II and sqrt(p/15) each of the other 15
  Pauli products;
* TwoQubitDephasing(p): sqrt(1-p) II and sqrt(p/3) each of IZ, ZI, ZZ;
* TwoQubitPauliChannel({"XY": p, ...}): sqrt(1-sum p) II and sqrt(p) per
  product;
* AmplitudeDamping(g): [[1, 0], [0, sqrt(1-g)]], [[0, sqrt(g)], [0, 0]];
* GeneralizedAmplitudeDamping(g, p): sqrt(p) times the two amplitude-damping
  operators, and sqrt(1-p) [[sqrt(1-g), 0], [0, 1]], sqrt(1-p) [[0, 0],
  [sqrt(g), 0]];
* PhaseDamping(g): [[1, 0], [0, sqrt(1-g)]], [[0, 0], [0, sqrt(g)]];
* Kraus(targets, matrices): the caller's operators (checked for sum K^H K = I).
A k-qubit operator's row/column index has targets[0] as its most
significant bit, as for gates.
"""
from __future__ import annotations

import itertools
from typing import Sequence

import numpy as np

_I = np.eye(2, dtype=np.complex128)
_X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
_Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
_Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)
_PAULI = {"I": _I, "X": _X, "Y": _Y, "Z": _Z}


class KrausChannel:
    """A completely positive trace-preserving map rho -> sum_i K_i rho K_i^H."""

    num_qubits = 1

    def __init__(self, targets: Sequence[int]):
        t = tuple(int(q) for q in targets)
        if len(t) != self.num_qubits or len(set(t)) != len(t):
            raise ValueError(f"{type(self).__name__} acts on {self.num_qubits} distinct qubit(s), got {t}")
        self._targets = t

    @property
    def targets(self) -> tuple[int, ...]:
        return self._targets

    @property
    def matrices(self) -> list[np.ndarray]:
        raise NotImplementedError

    def superoperator(self) -> np.ndarray:
        """sum_i K_i (x) conj(K_i): the channel on vec(rho) with row index
        (r, c) -> r * 2^k + c."""
        return sum(np.kron(k, np.conj(k)) for k in self.matrices)


def _probability(p: float, name: str = "probability", hi: float = 1.0) -> float:
    p = float(p)
    if not 0.0 <= p <= hi:
        raise ValueError(f"{name} must be in [0, {hi}], got {p}")
    return p


class BitFlip(KrausChannel):
    def __init__(self, targets, probability):
        super().__init__(targets)
        self.probability = _probability(probability)

    @property
    def matrices(self):
        p = self.probability
        return [np.sqrt(1 - p) * _I, np.sqrt(p) * _X]


class PhaseFlip(KrausChannel):
    def __init__(self, targets, probability):
        super().__init__(targets)
        self.probability = _probability(probability)

    @property
    def matrices(self):
        p = self.probability
        return [np.sqrt(1 - p) * _I, np.sqrt(p) * _Z]


class PauliChannel(KrausChannel):
    def __init__(self, targets, probX, probY, probZ):
        super().__init__(targets)
        self.probabilities = (_probability(probX), _probability(probY), _probability(probZ))
        _probability(sum(self.probabilities), "total probability")

    @property
    def matrices(self):
        px, py, pz = self.probabilities
        return [np.sqrt(1 - px - py - pz) * _I, np.sqrt(px) * _X, np.sqrt(py) * _Y, np.sqrt(pz) * _Z]


class Depolarizing(KrausChannel):
    def __init__(self, targets, probability):
        super().__init__(targets)
        self.probability = _probability(probability, hi=0.75)

    @property
    def matrices(self):
        p = self.probability
        return [np.sqrt(1 - p) * _I] + [np.sqrt(p / 3) * m for m in (_X, _Y, _Z)]


class TwoQubitDepolarizing(KrausChannel):
    num_qubits = 2

    def __init__(self, targets, probability):
        super().__init__(targets)
        self.probability = _probability(probability, hi=15 / 16)

    @property
    def matrices(self):
        p = self.probability
        out = []
        for a, b in itertools.product("IXYZ", repeat=2):
            w = np.sqrt(1 - p) if a + b == "II" else np.sqrt(p / 15)
            out.append(w * np.kron(_PAULI[a], _PAULI[b]))
        return out


class TwoQubitDephasing(KrausChannel):
    num_qubits = 2

    def __init__(self, targets, probability):
        super().__init__(targets)
        self.probability = _probability(probability, hi=0.75)

    @property
    def matrices(self):
        p = self.probability
        return [np.sqrt(1 - p) * np.kron(_I, _I)] + [
            np.sqrt(p / 3) * np.kron(_PAULI[a], _PAULI[b]) for a, b in ("IZ", "ZI", "ZZ")]


class TwoQubitPauliChannel(KrausChannel):
    num_qubits = 2

    def __init__(self, targets, probabilities: dict[str, float]):
        super().__init__(targets)
        for k in probabilities:
            if len(k) != 2 or set(k) - set("IXYZ") or k == "II":
                raise ValueError(f"bad two-qubit Pauli {k!r}")
        self.probabilities = {k: _probability(v) for k, v in probabilities.items()}
        _probability(sum(self.probabilities.values()), "total probability")

    @property
    def matrices(self):
        total = sum(self.probabilities.values())
        out = [np.sqrt(1 - total) * np.kron(_I, _I)]
        for k, p in self.probabilities.items():
            out.append(np.sqrt(p) * np.kron(_PAULI[k[0]], _PAULI[k[1]]))
        return out


class AmplitudeDamping(KrausChannel):
    def __init__(self, targets, gamma):
        super().__init__(targets)
        self.gamma = _probability(gamma, "gamma")

    @property
    def matrices(self):
        g = self.gamma
        return [np.array([[1, 0], [0, np.sqrt(1 - g)]], dtype=np.complex128),
                np.array([[0, np.sqrt(g)], [0, 0]], dtype=np.complex128)]


class GeneralizedAmplitudeDamping(KrausChannel):
    def __init__(self, targets, gamma, probability):
        super().__init__(targets)
        self.gamma = _probability(gamma, "gamma")
        self.probability = _probability(probability)

    @property
    def matrices(self):
        g, p = self.gamma, self.probability
        a, b = np.sqrt(p), np.sqrt(1 - p)
        return [a * np.array([[1, 0], [0, np.sqrt(1 - g)]], dtype=np.complex128),
                a * np.array([[0, np.sqrt(g)], [0, 0]], dtype=np.complex128),
                b * np.array([[np.sqrt(1 - g), 0], [0, 1]], dtype=np.complex128),
                b * np.array([[0, 0], [np.sqrt(g), 0]], dtype=np.complex128)]


class PhaseDamping(KrausChannel):
    def __init__(self, targets, gamma):
        super().__init__(targets)
        self.gamma = _probability(gamma, "gamma")

    @property
    def matrices(self):
        g = self.gamma
        return [np.array([[1, 0], [0, np.sqrt(1 - g)]], dtype=np.complex128),
                np.array([[0, 0], [0, np.sqrt(g)]], dtype=np.complex128)]


class Kraus(KrausChannel):
    def __init__(self, targets, matrices: Sequence[np.ndarray]):
        ms = [np.array(m, dtype=np.complex128) for m in matrices]
        if not ms:
            raise ValueError("Kraus needs at least one operator")
        d = ms[0].shape[0]
        if any(m.shape != (d, d) for m in ms) or d & (d - 1) or d < 2:
            raise ValueError("Kraus operators must be equal-sized 2^k x 2^k matrices")
        self.num_qubits = d.bit_length() - 1
        super().__init__(targets)
        if not np.allclose(sum(m.conj().T @ m for m in ms), np.eye(d), atol=1e-10):
            raise ValueError("Kraus operators do not sum to the identity (sum K^H K != I)")
        self._matrices = ms

    @property
    def matrices(self):
        return list(self._matrices)
