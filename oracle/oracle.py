"""ctypes bindings to the two C oracles, plus numpy restatements.

TEST ORACLE ONLY: see the package docstring for who may import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Iterable, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libsnuqs_ref.so")

# GateOperationType order (operation.h:17-52), then the gates the reference
# names but does not implement (gate_operations.py:238).
GATE_NAMES = [
    "Identity", "Hadamard", "PauliX", "PauliY", "PauliZ", "CX", "CY", "CZ",
    "S", "Si", "T", "Ti", "V", "Vi", "PhaseShift", "CPhaseShift",
    "CPhaseShift00", "CPhaseShift01", "CPhaseShift10", "RotX", "RotY", "RotZ",
    "Swap", "ISwap", "PSwap", "XY", "XX", "YY", "ZZ", "CCNot", "CSwap", "U",
    "GPhase", "SwapA2A", "ECR", "CV", "PRx",
]
GATE_ID = {n: i for i, n in enumerate(GATE_NAMES)}
REFERENCE_GATES = GATE_NAMES[:34]  # gates the reference constructs itself


def build() -> None:
    """Builds liboracle.so, and oracle/_ref when the reference sources exist."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load(path: str) -> ctypes.CDLL:
    if not os.path.exists(path):
        build()
    return ctypes.CDLL(path)


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = _load(_ORACLE_SO)
        dp, ip, i = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_int
        _lib.oracle_gate_matrix.argtypes = [i, dp, dp]
        _lib.oracle_gate_qubits.argtypes = [i]
        _lib.oracle_gate_num_angles.argtypes = [i]
        _lib.oracle_apply.argtypes = [dp, i, dp, ip, i]
        _lib.oracle_apply_gate.argtypes = [dp, i, i, ip, i, dp]
        _lib.oracle_initialize_basis_z.argtypes = [dp, i]
    return _lib


def ref_available() -> bool:
    """The compiled reference library exists, or its sources do (REF, as in
    the Makefile) so that build() can make it."""
    src = os.path.join(os.environ.get("REF", "/root/reference"), "src", "braket", "snuqs", "csrc")
    return os.path.exists(_REF_SO) or os.path.isdir(src)


def ref() -> ctypes.CDLL:
    """The reference's own CPU gate path (compiled from its sources)."""
    global _ref
    if _ref is None:
        _ref = _load(_REF_SO)
        dp, sp, s, i = (ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_size_t),
                        ctypes.c_size_t, ctypes.c_int)
        _ref.ref_gate_matrix.argtypes = [i, dp, s, dp]
        _ref.ref_apply_gate.argtypes = [dp, s, i, sp, s, dp]
        _ref.ref_apply_matrix.argtypes = [dp, s, dp, sp, s]
        _ref.ref_initialize_basis_z.argtypes = [dp, s]
        _ref.ref_max_threads.restype = ctypes.c_int
    return _ref


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def gate_qubits(name: str) -> int:
    return lib().oracle_gate_qubits(GATE_ID[name])


def gate_num_angles(name: str) -> int:
    return lib().oracle_gate_num_angles(GATE_ID[name])


def gate_matrix(name: str, angles: Sequence[float] = ()) -> np.ndarray:
    """Restated matrix of a named gate (2^k x 2^k complex128)."""
    k = gate_qubits(name)
    a = np.zeros(3, dtype=np.float64)
    a[: len(angles)] = angles
    out = np.zeros((1 << k, 1 << k), dtype=np.complex128)
    if lib().oracle_gate_matrix(GATE_ID[name], _dptr(a), _dptr(out)) < 0:
        raise ValueError(name)
    return out


def ref_gate_matrix(name: str, angles: Sequence[float] = ()) -> np.ndarray:
    """The reference constructor's own matrix (gate_operations.cc)."""
    k = gate_qubits(name)
    a = np.zeros(3, dtype=np.float64)
    a[: len(angles)] = angles
    out = np.zeros((1 << k, 1 << k), dtype=np.complex128)
    if ref().ref_gate_matrix(GATE_ID[name], _dptr(a), k, _dptr(out)) != 0:
        raise ValueError(name)
    return out


def ref_initialize_basis_z(state: np.ndarray, nq: int) -> None:
    """In place: the reference cpu::initializeBasis_Z on a host state."""
    assert state.dtype == np.complex128 and state.size == (1 << nq)
    ref().ref_initialize_basis_z(_dptr(state), nq)


def basis_state(nq: int, index: int = 0) -> np.ndarray:
    s = np.zeros(1 << nq, dtype=np.complex128)
    s[index] = 1.0
    return s


def apply_matrix(state: np.ndarray, nq: int, matrix: np.ndarray,
                 targets: Sequence[int]) -> None:
    """In place: cpu::applyGate restated, any k."""
    assert state.dtype == np.complex128 and state.flags.c_contiguous
    m = np.ascontiguousarray(matrix, dtype=np.complex128)
    t = (ctypes.c_int * max(1, len(targets)))(*targets)
    if lib().oracle_apply(_dptr(state), nq, _dptr(m), t, len(targets)) != 0:
        raise ValueError("oracle_apply failed")


def ref_apply_matrix(state: np.ndarray, nq: int, matrix: np.ndarray,
                     targets: Sequence[int]) -> None:
    """In place: the reference cpu::applyGate with this matrix (k <= 3)."""
    m = np.ascontiguousarray(matrix, dtype=np.complex128)
    t = (ctypes.c_size_t * max(1, len(targets)))(*targets)
    if ref().ref_apply_matrix(_dptr(state), nq, _dptr(m), t, len(targets)) != 0:
        raise ValueError("ref_apply_matrix failed")


def ref_apply_gate(state: np.ndarray, nq: int, name: str, targets: Sequence[int],
                   angles: Sequence[float] = ()) -> None:
    """In place: the reference gate constructor + cpu::applyGate."""
    a = np.zeros(3, dtype=np.float64)
    a[: len(angles)] = angles
    t = (ctypes.c_size_t * max(1, len(targets)))(*targets)
    if ref().ref_apply_gate(_dptr(state), nq, GATE_ID[name], t, len(targets), _dptr(a)) != 0:
        raise ValueError(name)


def run_ops(ops: Iterable, nq: int, state: np.ndarray | None = None,
            use_ref: bool = False) -> np.ndarray:
    """Runs (name, targets, angles[, matrix]) ops from |0..0> (or `state`).

    ``name == "Unitary"`` carries its matrix as the 4th element.  With
    ``use_ref`` the reference CPU library applies every gate it has (Unitary
    through cpu::applyGate with the caller's matrix, k <= 3); otherwise the C
    restatement does.
    """
    psi = basis_state(nq) if state is None else np.array(state, dtype=np.complex128)
    for op in ops:
        name, targets, angles = op[0], list(op[1]), list(op[2])
        if name == "Unitary":
            m = op[3]
            (ref_apply_matrix if use_ref else apply_matrix)(psi, nq, m, targets)
        elif use_ref and name in REFERENCE_GATES:
            ref_apply_gate(psi, nq, name, targets, angles)
        elif use_ref:
            ref_apply_matrix(psi, nq, gate_matrix(name, angles), targets)
        else:
            apply_matrix(psi, nq, gate_matrix(name, angles), targets)
    return psi


# ---------------------------------------------------------------------------
# Gate reordering: transpile.py:33-54 (pseudo_gt) and :74-89
# (pseudo_sort_operations_descending).  GateOperation.sliceable() is always
# False in the reference (operation.cc:175), so its branches never fire.
# ---------------------------------------------------------------------------
def _pseudo_gt(t1: Sequence[int], p1: int, t2: Sequence[int], p2: int) -> bool:
    if len(t1) == 0 and len(t2) == 0:
        return p1 < p2
    if len(t1) == 0:
        return True
    if len(t2) == 0:
        return False
    if set(t1) & set(t2):
        return p1 < p2
    return min(t1) > min(t2)


def pseudo_sort_descending(targets_list: Sequence[Sequence[int]]) -> list[int]:
    """Returns the permutation (old indices in new order) the reference's
    insertion sort produces.  Positions compared are the ORIGINAL indices i
    (of the element being inserted) and j (the slot it is compared with), as
    the reference passes them (transpile.py:82-83)."""
    order = list(range(len(targets_list)))
    for i in range(1, len(order)):
        cur = order[i]
        j = i - 1
        while j >= 0:
            other = order[j]
            if _pseudo_gt(targets_list[cur], i, targets_list[other], j):
                order[j + 1] = order[j]
            else:
                break
            j -= 1
        if i != j + 1:
            order[j + 1] = cur
    return order


# ---------------------------------------------------------------------------
# Result restatements (numpy).  Qubit q is index bit nq-1-q.
# ---------------------------------------------------------------------------
def probabilities(state: np.ndarray) -> np.ndarray:
    """simulation.py:208-215: |psi|^2."""
    return np.abs(state) ** 2


_PAULI = {
    "I": np.eye(2, dtype=np.complex128),
    "X": np.array([[0, 1], [1, 0]], dtype=np.complex128),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    "Z": np.array([[1, 0], [0, -1]], dtype=np.complex128),
}


def apply_pauli_string(state: np.ndarray, nq: int, pauli: str) -> np.ndarray:
    """P|psi> for a Pauli string whose character q acts on qubit q
    (observables.py PauliX/Y/Z + TensorProduct semantics)."""
    psi = np.asarray(state, dtype=np.complex128).reshape([2] * nq)
    for q, ch in enumerate(pauli):
        if ch == "I":
            continue
        psi = np.moveaxis(np.tensordot(_PAULI[ch], psi, axes=([1], [q])), 0, q)
    return psi.reshape(-1)


def expectation(state: np.ndarray, nq: int, terms: Sequence[tuple[float, str]]) -> float:
    """sum_t w_t <psi|P_t|psi> (real part), FP64."""
    total = 0.0
    for w, p in terms:
        total += w * float(np.real(np.vdot(state, apply_pauli_string(state, nq, p))))
    return total


# ---------------------------------------------------------------------------
# Measurement sampling (restates the device sampler's definition; the
# reference samples with np.random.choice over |psi|^2, simulation.py:216-220,
# whose random stream cannot be reproduced on the device).
# ---------------------------------------------------------------------------
SAMPLE_LEAF_BITS = 12


def probability_tree(state: np.ndarray) -> list:
    """Levels of the fixed binary tree of FP64 probability sums: level d has
    2^d nodes, the last level is |psi_i|^2 (padded with zeros to at least
    2^12 entries); each node is the IEEE sum of its two children."""
    a = np.asarray(state).astype(np.complex128, copy=False)
    p = a.real * a.real + a.imag * a.imag  # two products and one sum, no fused multiply-add
    size = max(p.size, 1 << SAMPLE_LEAF_BITS)
    if size != p.size:
        p = np.concatenate([p, np.zeros(size - p.size)])
    levels = [p]
    while levels[-1].size > 1:
        x = levels[-1]
        levels.append(x[0::2] + x[1::2])
    levels.reverse()
    return levels


def sample_inverse_cdf(state: np.ndarray, uniforms: np.ndarray) -> np.ndarray:
    """Shot s: r = u_s * total; walk the tree from the root, going left when
    r < left sum or the right sum is 0, else r -= left sum and go right."""
    levels = probability_tree(state)
    u = np.asarray(uniforms, dtype=np.float64)
    r = u * levels[0][0]
    k = np.zeros(u.size, dtype=np.int64)
    for d in range(1, len(levels)):
        lv = levels[d]
        left_sum, right_sum = lv[2 * k], lv[2 * k + 1]
        left = (r < left_sum) | (right_sum == 0.0)
        r = np.where(left, r, r - left_sum)
        k = 2 * k + (~left).astype(np.int64)
    return k.astype(np.uint64)


def marginal_probabilities(state: np.ndarray, nq: int, qubits: Sequence[int]) -> np.ndarray:
    """Probabilities of the basis states of `qubits` (qubits[0] most
    significant), the others traced out."""
    p = (np.abs(np.asarray(state, dtype=np.complex128)) ** 2).reshape([2] * nq)
    rest = [q for q in range(nq) if q not in qubits]
    m = p.sum(axis=tuple(rest)) if rest else p
    # Remaining axes are in ascending qubit order; put them in `qubits` order.
    order = sorted(qubits)
    m = np.transpose(m, [order.index(q) for q in qubits]) if len(qubits) > 1 else m
    return np.asarray(m).reshape(-1)


def variance(state: np.ndarray, nq: int, terms: Sequence[tuple[float, str]]) -> float:
    """<H^2> - <H>^2 with H = sum_t w_t P_t: |H psi|^2 - <psi|H psi>^2."""
    h = np.zeros_like(np.asarray(state, dtype=np.complex128))
    for w, pstr in terms:
        h += w * apply_pauli_string(state, nq, pstr)
    e1 = float(np.real(np.vdot(state, h)))
    return float(np.real(np.vdot(h, h))) - e1 * e1


def expectation_indexed(state: np.ndarray, nq: int, terms: Sequence[tuple[float, str]]) -> float:
    """The same sum_t w_t <psi|P_t|psi> as `expectation`, by index arithmetic
    (P|i> = i^ny (-1)^popc(i & z) |i ^ x> for flip mask x, Z-or-Y mask z and
    ny Y factors), for larger states."""
    psi = np.asarray(state, dtype=np.complex128)
    idx = np.arange(psi.size, dtype=np.uint64)
    groups: dict = {}
    for w, p in terms:
        x = z = 0
        ny = 0
        for q, ch in enumerate(p):
            bit = 1 << (nq - 1 - q)
            if ch in "XY":
                x |= bit
            if ch in "ZY":
                z |= bit
            ny += ch == "Y"
        groups.setdefault(x, []).append((w, z, ny))
    total = 0.0
    for x, ts in groups.items():
        prod = np.conj(psi) * psi[idx ^ np.uint64(x)]  # conj(psi_i) psi_(i^x)
        for w, z, ny in ts:
            sign = 1.0 - 2.0 * (np.bitwise_count(idx & np.uint64(z)) & 1)
            # <psi|P|psi> = sum_i conj(psi_i) (P psi)_i with (P psi)_i = i^ny (-1)^popc((i^x)&z) psi_(i^x)
            sign_shift = -1.0 if (bin(x & z).count("1") & 1) else 1.0
            val = (1j ** ny) * sign_shift * np.dot(sign, prod)
            total += w * float(np.real(val))
    return total


# ---------------------------------------------------------------------------
# Density matrices (noise channels; the reference defines Kraus channels in
# noise_operations.py but never simulates them).
# ---------------------------------------------------------------------------
def _apply_left(rho: np.ndarray, nq: int, m: np.ndarray, targets: Sequence[int]) -> np.ndarray:
    """m (on `targets`) times rho: m applied to every column of rho."""
    out = np.array(rho, dtype=np.complex128, order="F")
    for j in range(out.shape[1]):
        col = np.ascontiguousarray(out[:, j])
        apply_matrix(col, nq, m, targets)
        out[:, j] = col
    return out


def density_evolve(nq: int, steps) -> np.ndarray:
    """rho after `steps`, each ("unitary", matrix, targets) or ("kraus",
    [K_i], targets), from |0...0><0...0|: rho -> U rho U^H and
    rho -> sum_i K_i rho K_i^H, each product formed column by column."""
    d = 1 << nq
    rho = np.zeros((d, d), dtype=np.complex128)
    rho[0, 0] = 1.0
    for kind, mats, targets in steps:
        ks = [mats] if kind == "unitary" else mats
        new = np.zeros_like(rho)
        for k in ks:
            kr = _apply_left(rho, nq, k, targets)                   # K rho
            new += _apply_left(kr.conj().T, nq, k, targets).conj().T  # (K (K rho)^H)^H
        rho = new
    return rho
