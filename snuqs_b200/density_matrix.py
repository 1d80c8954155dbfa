"""Noisy circuits as density matrices on the engine.

A density matrix rho of n qubits is held as a 2n-qubit engine state v with
v[(r << n) | c] = rho[r, c]: qubit q of the row index is engine qubit q and
qubit q of the column index is engine qubit n + q.  Then
* a gate U on targets T: rho -> U rho U^H is U on qubits T and conj(U) on
  qubits n + T (two queued gates; the planner fuses them into the same
  sweeps as any other gates);
* a Kraus channel {K_i} on T: rho -> sum_i K_i rho K_i^H is the dense
  superoperator sum_i K_i (x) conj(K_i) on qubits T + (n + T), one queued
  2k-qubit matrix;
* probabilities are the diagonal rho[i, i] = v[i (2^n + 1)], and
  Tr(P rho) for a Pauli string P = i^ny X^x Z^z is
  sum_c i^ny (-1)^popc(c & z) rho[c, c ^ x], both gathered on the device
  (sq_amplitudes) at 2^n entries per flip group.
The reference defines noise channels (src/braket/snuqs/noise_operations.py)
but its simulator refuses them (src/braket/snuqs/simulator.py:650-659).
A complex128 density matrix of n qubits takes 16 * 4^n bytes: 16 qubits fill
64 GiB.
"""
from __future__ import annotations

from typing import Iterable, Optional, Sequence

import numpy as np

from . import capi, circuits
from .noise_operations import KrausChannel


class DensityMatrixSimulation:
    def __init__(self, qubit_count: int, shots: int = 0, precision: str = "complex128",
                 seed: Optional[int] = None, stream=None):
        if precision not in ("complex128", "complex64"):
            raise ValueError("precision must be 'complex128' or 'complex64'")
        if qubit_count < 2 or qubit_count > 17:
            raise ValueError("density matrices of 2..17 qubits")
        self._n = int(qubit_count)
        self._shots = int(shots)
        dtype = capi.SQ_C128 if precision == "complex128" else capi.SQ_C64
        self._state = capi.State(2 * self._n, dtype, stream=stream)
        self._state.init_basis(0)  # |0...0><0...0|
        self._rng = np.random.default_rng(seed)

    @property
    def qubit_count(self) -> int:
        return self._n

    @property
    def shots(self) -> int:
        return self._shots

    @property
    def engine_state(self) -> capi.State:
        return self._state

    def _gate(self, m: np.ndarray, targets: Sequence[int]) -> None:
        if len(targets) == 0:
            return  # a global phase cancels in U rho U^H
        n = self._n
        self._state.apply_matrix(m, list(targets))
        self._state.apply_matrix(np.conj(m), [n + q for q in targets])

    def evolve(self, operations: Iterable) -> None:
        n = self._n
        for op in operations:
            if isinstance(op, KrausChannel):
                t = list(op.targets)
                self._state.apply_matrix(op.superoperator(), t + [n + q for q in t])
            elif isinstance(op, tuple):
                self._gate(circuits.op_matrix(op, capi.gate_matrix), op[1])
            else:  # a _C GateOperation
                self._gate(np.array(op, dtype=np.complex128), list(op.targets))

    @property
    def density_matrix(self) -> np.ndarray:
        d = 1 << self._n
        return self._state.to_host().reshape(d, d)

    @property
    def probabilities(self) -> np.ndarray:
        d = 1 << self._n
        return self._state.amplitudes(np.arange(d, dtype=np.int64) * (d + 1)).real.copy()

    def expectation(self, terms: Sequence[tuple[float, str]]) -> float:
        """Tr(H rho) for H = sum_t w_t P_t (Pauli strings, character q on qubit q)."""
        n = self._n
        d = 1 << n
        c = np.arange(d, dtype=np.int64)
        groups: dict = {}
        for w, p in terms:
            if len(p) != n:
                raise ValueError("Pauli string length must equal the qubit count")
            x = z = ny = 0
            for q, ch in enumerate(p):
                bit = 1 << (n - 1 - q)
                x |= bit if ch in "XY" else 0
                z |= bit if ch in "ZY" else 0
                ny += ch == "Y"
            groups.setdefault(x, []).append((w, z, ny))
        total = 0.0
        for x, ts in groups.items():
            g = self._state.amplitudes((c << n) | (c ^ x))  # rho[c, c ^ x]
            for w, z, ny in ts:
                sign = 1.0 - 2.0 * (np.bitwise_count((c & z).astype(np.uint64)) & 1)
                total += w * float(np.real((1j ** ny) * np.dot(sign, g)))
        return total

    def trace(self) -> float:
        return float(self.probabilities.sum())

    def retrieve_samples(self) -> np.ndarray:
        """`shots` basis-state indices drawn from the diagonal of rho."""
        if self._shots == 0:
            return np.array([], dtype=np.int64)
        p = np.clip(self.probabilities, 0.0, None)
        cdf = np.cumsum(p)
        u = self._rng.random(self._shots) * cdf[-1]
        return np.minimum(np.searchsorted(cdf, u, side="right"), p.size - 1).astype(np.int64)

    def close(self) -> None:
        if self._state is not None:
            self._state.close()
            self._state = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
