"""State-vector simulation on the engine: the reference plugin's
StateVectorSimulation (src/braket/snuqs/simulation.py:80-542) for its
no-offload CUDA path, re-based on the C ABI.

What the reference does per run, and what replaces it here:
* initialise a CUDA StateVector and initialize_basis_z (:117-122) --
  `StateVectorSimulation(qubit_count, shots)` creates an sq_state in |0...0>;
* evolve: pseudo-sort the operations, then one functionals.apply per gate in
  a Python loop (:274-284) -- `evolve(operations)` queues every gate and runs
  them as fused sweeps at the next result (the engine reorders commuting
  gates itself);
* state_vector / probabilities: a full device-to-host copy and |psi|^2 in
  numpy (:195-214) -- `state_vector` still copies (it is the state), but
  `probabilities` is computed on the device and `retrieve_samples` (:216-220:
  np.random.choice over the copied probabilities) runs the device sampler and
  copies back only the shot indices.

Operations are (name, targets, angles[, matrix]) tuples, a Unitary carrying
its matrix, or _C.operation.GateOperation objects (their matrix and
targets, with ctrl_modifiers/power already applied by _C).
"""
from __future__ import annotations

from typing import Iterable, Optional

import numpy as np

from . import capi


class StateVectorSimulation:
    def __init__(self, qubit_count: int, shots: int = 0, precision: str = "complex128",
                 seed: Optional[int] = None, stream=None):
        if precision not in ("complex128", "complex64"):
            raise ValueError("precision must be 'complex128' or 'complex64'")
        self._qubit_count = int(qubit_count)
        self._shots = int(shots)
        self._dtype = capi.SQ_C128 if precision == "complex128" else capi.SQ_C64
        self._state = capi.State(self._qubit_count, self._dtype, stream=stream)
        self._state.init_basis(0)
        self._rng = np.random.default_rng(seed)
        self._operations: list = []

    # -- Simulation surface (simulation.py:14-77) ---------------------------
    @property
    def qubit_count(self) -> int:
        return self._qubit_count

    @property
    def shots(self) -> int:
        return self._shots

    @property
    def precision(self) -> str:
        return "complex64" if self._dtype == capi.SQ_C64 else "complex128"

    @property
    def engine_state(self) -> capi.State:
        """The engine's state handle (for result types)."""
        return self._state

    @property
    def operations(self) -> list:
        """Every operation evolved so far, in order (for adjoint gradients)."""
        return list(self._operations)

    def evolve(self, operations: Iterable) -> None:
        for op in operations:
            if isinstance(op, tuple):
                if op[0] == "Unitary":
                    self._state.apply_matrix(op[3], op[1])
                else:
                    self._state.apply_gate(op[0], op[1], op[2])
            else:  # a _C GateOperation: buffer protocol gives its matrix
                m = np.array(op, copy=False)
                self._state.apply_matrix(np.ascontiguousarray(m, dtype=np.complex128), list(op.targets))
            self._operations.append(op)

    @property
    def state_vector(self) -> np.ndarray:
        return self._state.to_host()

    @property
    def probabilities(self) -> np.ndarray:
        return self._state.marginal_probabilities(list(range(self._qubit_count)))

    def retrieve_samples(self) -> np.ndarray:
        """`shots` basis-state indices drawn from |psi|^2 on the device."""
        if self._shots == 0:
            return np.array([], dtype=np.int64)
        u = self._rng.random(self._shots)
        return self._state.sample(u).astype(np.int64)

    def close(self) -> None:
        if self._state is not None:
            self._state.close()
            self._state = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
