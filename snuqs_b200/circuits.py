"""Seeded synthetic circuits with the shapes of the reference's benchmarks.

Ops are tuples ``(name, qubits, angles)``; ``("Unitary", qubits, (), matrix)``
carries its matrix.  Names are the reference's gate class names
(``src/braket/snuqs/csrc/operation/gate_operations.h``).  Every generator
takes a seed and draws from ``numpy.random.default_rng(seed)``; no public
benchmark items are used, only the circuit shapes:

* GHZ ladder (``benchmark/ghz.py:53-58``),
* quantum-volume layers of Haar-random 4x4 unitaries on a random pairing
  (``benchmark/quantum_volume.py:30-46``),
* a hardware-efficient VQE ansatz of RY/RZ layers and a CX ladder
  (``benchmark/vqe.py:52-76``),
* QAOA MaxCut on a random 3-regular graph,
* the uniform random gate mix of ``test/braket/test_random_circuit.py:10-117``.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

TWO_PI = 2.0 * np.pi

# Gate name -> (qubits, angles); the reference's 33 Python-bound gates
# (pymodule.cc:88-120) plus the Braket gates it dropped.
GATES = {
    "Identity": (1, 0), "Hadamard": (1, 0), "PauliX": (1, 0), "PauliY": (1, 0),
    "PauliZ": (1, 0), "CX": (2, 0), "CY": (2, 0), "CZ": (2, 0), "S": (1, 0),
    "Si": (1, 0), "T": (1, 0), "Ti": (1, 0), "V": (1, 0), "Vi": (1, 0),
    "PhaseShift": (1, 1), "CPhaseShift": (2, 1), "CPhaseShift00": (2, 1),
    "CPhaseShift01": (2, 1), "CPhaseShift10": (2, 1), "RotX": (1, 1),
    "RotY": (1, 1), "RotZ": (1, 1), "Swap": (2, 0), "ISwap": (2, 0),
    "PSwap": (2, 1), "XY": (2, 1), "XX": (2, 1), "YY": (2, 1), "ZZ": (2, 1),
    "CCNot": (3, 0), "CSwap": (3, 0), "U": (1, 3), "GPhase": (0, 1),
    "ECR": (2, 0), "CV": (2, 0), "PRx": (1, 2),
}
# The 33 gates test_random_circuit.py draws from (lines 13-47).
REFERENCE_TEST_GATES = [
    "Identity", "Hadamard", "PauliX", "PauliY", "PauliZ", "CX", "CY", "CZ", "S",
    "Si", "T", "Ti", "V", "Vi", "PhaseShift", "CPhaseShift", "CPhaseShift00",
    "CPhaseShift01", "CPhaseShift10", "RotX", "RotY", "RotZ", "Swap", "ISwap",
    "PSwap", "XY", "XX", "YY", "ZZ", "CCNot", "CSwap", "U", "GPhase",
]
# The random-mix workload: 14 gate types drawn uniformly.
MIX_GATES = ["RotX", "RotY", "RotZ", "U", "PhaseShift",
             "CX", "CZ", "Swap", "ISwap", "XX", "YY", "ZZ",
             "CCNot", "CSwap"]


def _draw(rng: np.random.Generator, n: int, names: Sequence[str], ngates: int) -> list:
    ops = []
    for _ in range(ngates):
        name = names[int(rng.integers(len(names)))]
        k, na = GATES[name]
        qubits = tuple(int(q) for q in rng.choice(n, size=k, replace=False)) if k else ()
        angles = tuple(float(a) for a in rng.uniform(0.0, TWO_PI, size=na))
        ops.append((name, qubits, angles))
    return ops


def ghz(n: int) -> list:
    """H(0) then CX(i, i+1), i = 0..n-2, from |0...0>."""
    return [("Hadamard", (0,), ())] + [("CX", (i, i + 1), ()) for i in range(n - 1)]


def random_mix(n: int, ngates: int = 400, seed: int = 1234) -> list:
    """Uniform draws from the 14-gate mix; distinct random qubits; angles
    uniform in [0, 2pi)."""
    return _draw(np.random.default_rng(seed), n, MIX_GATES, ngates)


def random_all_gates(n: int, ngates: int, seed: int = 1234, names: Sequence[str] | None = None) -> list:
    """H on every qubit, then `ngates` uniform draws over the reference
    test's 33 gates (test_random_circuit.py:113-117), seeded."""
    rng = np.random.default_rng(seed)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    return ops + _draw(rng, n, list(names or REFERENCE_TEST_GATES), ngates)


def haar_unitary(d: int, rng: np.random.Generator) -> np.ndarray:
    """Haar-random d x d unitary: QR of a complex Gaussian, with Q's columns
    multiplied by diag(R)/|diag(R)| (Mezzadri's phase fix)."""
    z = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    ph = np.diag(r) / np.abs(np.diag(r))
    return q * ph[None, :]


def quantum_volume(n: int, depth: int | None = None, seed: int = 1234) -> list:
    """`depth` layers; each pairs the qubits by a random permutation and
    applies a Haar 4x4 Unitary to each pair."""
    rng = np.random.default_rng(seed)
    depth = n if depth is None else depth
    ops = []
    for _ in range(depth):
        perm = rng.permutation(n)
        for w in range(n // 2):
            u = haar_unitary(4, rng)
            ops.append(("Unitary", (int(perm[2 * w]), int(perm[2 * w + 1])), (), u))
    return ops


def vqe_ansatz(n: int, angles: np.ndarray | None = None, layers: int = 6, seed: int = 1234) -> list:
    """`layers` x (RY on every qubit, RZ on every qubit, CX(i, i+1) ladder)."""
    if angles is None:
        angles = np.random.default_rng(seed).uniform(0.0, TWO_PI, size=2 * n * layers)
    ops, p = [], 0
    for _ in range(layers):
        for q in range(n):
            ops.append(("RotY", (q,), (float(angles[p]),)))
            p += 1
        for q in range(n):
            ops.append(("RotZ", (q,), (float(angles[p]),)))
            p += 1
        for q in range(n - 1):
            ops.append(("CX", (q, q + 1), ()))
    return ops


def random_pauli_hamiltonian(n: int, nterms: int = 64, seed: int = 1234):
    """`nterms` random Pauli strings (I/X/Y/Z uniform per qubit) with N(0,1)
    weights: list of (weight, string)."""
    rng = np.random.default_rng(seed)
    letters = np.array(list("IXYZ"))
    return [(float(rng.standard_normal()), "".join(letters[rng.integers(4, size=n)]))
            for _ in range(nterms)]


def random_regular_graph(n: int, d: int = 3, seed: int = 1234) -> list:
    """Seeded random d-regular simple graph (configuration model with
    restarts): list of edges (i, j), i < j."""
    rng = np.random.default_rng(seed)
    for _ in range(10000):
        stubs = np.repeat(np.arange(n), d)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        edges = set()
        ok = True
        for a, b in pairs:
            a, b = int(min(a, b)), int(max(a, b))
            if a == b or (a, b) in edges:
                ok = False
                break
            edges.add((a, b))
        if ok:
            return sorted(edges)
    raise RuntimeError("could not draw a simple regular graph")


def qaoa_maxcut(n: int, edges: Sequence, gammas: Sequence[float], betas: Sequence[float]) -> list:
    """H on every qubit, then p layers of ZZ(gamma_l) on each edge and
    RotX(beta_l) on each qubit.  Parameter index of every rotation:
    gamma_l -> l, beta_l -> p + l (see qaoa_param_map)."""
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for g, b in zip(gammas, betas):
        ops += [("ZZ", (int(i), int(j)), (float(g),)) for i, j in edges]
        ops += [("RotX", (q,), (float(b),)) for q in range(n)]
    return ops


def maxcut_hamiltonian(n: int, edges: Sequence):
    """<H_cost> = sum over edges of <Z_i Z_j> (weight +1 per edge; the cut
    value is (|E| - <H>)/2)."""
    terms = []
    for i, j in edges:
        s = ["I"] * n
        s[i] = s[j] = "Z"
        terms.append((1.0, "".join(s)))
    return terms


def op_matrix(op, gate_matrix) -> np.ndarray:
    """Matrix of an op tuple, using `gate_matrix(name, angles)` for named gates."""
    if op[0] == "Unitary":
        return np.asarray(op[3], dtype=np.complex128)
    return gate_matrix(op[0], op[2])
