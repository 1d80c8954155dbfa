"""Braket result types computed on the device.

Mirrors the reference plugin's result_types.py
(src/braket/snuqs/result_types.py: ResultType :32, TargetedResultType :56,
ObservableResultType :75, StateVector :132, from_braket_result_type :11),
which registers StateVector only (:149-151) while its simulator advertises
only that type (src/braket/snuqs/simulator.py:578-580) and forbids
Expectation, Variance, Probability, Amplitude and AdjointGradient
(:642-649).  Here every one of them is a device computation on the
simulation's resident state:

* Expectation / Variance -- the observable as a Pauli sum
  (snuqs_b200.observables), sq_expect_pauli / sq_variance_pauli;
* Probability -- sq_marginal_probabilities over the targets;
* Amplitude -- sq_amplitudes at the requested basis states;
* AdjointGradient -- sq_adjoint_gradient over the simulation's parametrised
  operations (one forward and one reverse pass).

As in the reference, an observable without targets yields one value per
qubit (ObservableResultType.calculate, result_types.py:97-115).  A front end
registers these with `from_braket_result_type`; the Braket IR types are
registered when the braket SDK is importable.
"""
from __future__ import annotations

from abc import ABC, abstractmethod
from functools import singledispatch
from typing import Any, Optional, Sequence, Union

import numpy as np

from . import observables as obs
from .simulation import StateVectorSimulation


class ResultType(ABC):
    @abstractmethod
    def calculate(self, simulation: StateVectorSimulation) -> Any:
        """The result on the simulation's current state."""


class TargetedResultType(ResultType, ABC):
    def __init__(self, targets: Optional[Sequence[int]] = None):
        self._targets = None if targets is None else tuple(int(t) for t in targets)

    @property
    def targets(self) -> Optional[tuple[int, ...]]:
        return self._targets


class ObservableResultType(TargetedResultType, ABC):
    def __init__(self, observable: obs.Observable):
        super().__init__(observable.measured_qubits)
        self._observable = observable

    @property
    def observable(self) -> obs.Observable:
        return self._observable

    @property
    def targets(self) -> Optional[tuple[int, ...]]:
        return self._observable.measured_qubits

    def calculate(self, simulation: StateVectorSimulation) -> Union[float, list[float]]:
        if self._observable.measured_qubits:
            return self._single(simulation, self._observable)
        return [self._single(simulation, self._observable.fix_qubit(q))
                for q in range(simulation.qubit_count)]

    @staticmethod
    @abstractmethod
    def _single(simulation: StateVectorSimulation, observable: obs.Observable) -> float:
        ...


class StateVector(ResultType):
    def calculate(self, simulation: StateVectorSimulation) -> np.ndarray:
        return simulation.state_vector


class Expectation(ObservableResultType):
    @staticmethod
    def _single(simulation, observable):
        return simulation.engine_state.expectation(observable.pauli_terms(simulation.qubit_count))


class Variance(ObservableResultType):
    @staticmethod
    def _single(simulation, observable):
        return simulation.engine_state.variance(observable.pauli_terms(simulation.qubit_count))


class Probability(TargetedResultType):
    """Probabilities of the basis states of the targets (all qubits when
    none), targets[0] the most significant bit."""

    def calculate(self, simulation: StateVectorSimulation) -> np.ndarray:
        qs = list(self._targets) if self._targets else list(range(simulation.qubit_count))
        return simulation.engine_state.marginal_probabilities(qs)


class Amplitude(ResultType):
    """Amplitudes of basis states given as bitstrings (character q is qubit q)."""

    def __init__(self, states: Sequence[str]):
        if not states:
            raise ValueError("Amplitude needs at least one basis state")
        self._states = list(states)

    @property
    def states(self) -> list[str]:
        return list(self._states)

    def calculate(self, simulation: StateVectorSimulation) -> dict[str, complex]:
        n = simulation.qubit_count
        for s in self._states:
            if len(s) != n or set(s) - {"0", "1"}:
                raise ValueError(f"basis state {s!r} is not a {n}-bit string")
        amps = simulation.engine_state.amplitudes([int(s, 2) for s in self._states])
        return {s: complex(a) for s, a in zip(self._states, amps)}


class AdjointGradient(ObservableResultType):
    """<observable> and its gradient with respect to the circuit parameters.

    The simulation's operations are (name, qubits, angles, params[, scales])
    tuples (params[j]: index of the parameter angle j follows, -1 =
    constant); `parameters` are the values of those parameters and
    `parameter_names` their names in the output (default "p0", "p1", ...)."""

    def __init__(self, observable: obs.Observable, parameters: Sequence[float],
                 parameter_names: Optional[Sequence[str]] = None):
        super().__init__(observable)
        self._theta = np.asarray(parameters, dtype=np.float64)
        self._names = list(parameter_names) if parameter_names is not None else \
            [f"p{i}" for i in range(self._theta.size)]
        if len(self._names) != self._theta.size:
            raise ValueError("one name per parameter")

    def calculate(self, simulation: StateVectorSimulation) -> dict:
        from . import adjoint

        if not self._observable.measured_qubits:
            raise ValueError("AdjointGradient needs a targeted observable")
        terms = self._observable.pauli_terms(simulation.qubit_count)
        ops = [op for op in simulation.operations if isinstance(op, tuple)]
        if len(ops) != len(simulation.operations):
            raise ValueError("AdjointGradient needs the circuit as operation tuples")
        ws = adjoint.Workspace(simulation.qubit_count, simulation.engine_state.dtype)
        try:
            e, g = adjoint.adjoint_gradient(ws, ops, self._theta, terms, self._theta.size)
        finally:
            ws.close()
        return {"expectation": e, "gradient": {k: float(v) for k, v in zip(self._names, g)}}

    @staticmethod
    def _single(simulation, observable):  # pragma: no cover - calculate() is overridden
        raise NotImplementedError


def from_braket_result_type(result_type) -> ResultType:
    """The ResultType for a Braket IR result type (reference :11-24)."""
    return _from_braket_result_type(result_type)


@singledispatch
def _from_braket_result_type(result_type):
    raise NotImplementedError(f"Result type {result_type} not recognized")


def from_braket_observable(ir_observable, ir_targets: Optional[Sequence[int]] = None) -> obs.Observable:
    """A Braket IR observable (list of factor names or matrices) as an
    Observable (reference _from_braket_observable, result_types.py:154-168)."""
    targets = list(ir_targets) if ir_targets else None

    def single(factor, tgts, is_factor=False):
        if isinstance(factor, str):
            cls = {"x": obs.PauliX, "y": obs.PauliY, "z": obs.PauliZ, "h": obs.Hadamard,
                   "i": obs.Identity}[factor.lower()]
            t = [tgts.pop(0)] if (tgts and is_factor) else (tgts if tgts else None)
            return cls(t)
        m = np.array(factor, dtype=np.float64)
        m = m[..., 0] + 1j * m[..., 1]
        k = int(m.shape[0]).bit_length() - 1
        if tgts and is_factor:
            t = [tgts.pop(0) for _ in range(k)]
        else:
            t = tgts if tgts else None
        return obs.Hermitian(m, t)

    if len(ir_observable) == 1:
        return single(ir_observable[0], targets)
    tg = list(targets) if targets else []
    factors = [single(f, tg, is_factor=True) for f in ir_observable]
    if tg:
        raise ValueError(f"Found {len(tg)} more target qubits than the tensor product acts on")
    return obs.TensorProduct(factors)


try:  # Braket IR registrations, when the SDK is present
    from braket.ir import jaqcd as _jaqcd

    @_from_braket_result_type.register
    def _(_: _jaqcd.StateVector):
        return StateVector()

    @_from_braket_result_type.register
    def _(rt: _jaqcd.Expectation):
        return Expectation(from_braket_observable(rt.observable, rt.targets))

    @_from_braket_result_type.register
    def _(rt: _jaqcd.Variance):
        return Variance(from_braket_observable(rt.observable, rt.targets))

    @_from_braket_result_type.register
    def _(rt: _jaqcd.Probability):
        return Probability(rt.targets)

    @_from_braket_result_type.register
    def _(rt: _jaqcd.Amplitude):
        return Amplitude(rt.states)
except Exception:  # noqa: BLE001 - the SDK is optional
    pass

SUPPORTED_RESULT_TYPES = [
    {"name": "StateVector", "observables": None, "minShots": 0, "maxShots": 0},
    {"name": "Expectation", "observables": ["x", "y", "z", "h", "i", "hermitian"], "minShots": 0,
     "maxShots": 0},
    {"name": "Variance", "observables": ["x", "y", "z", "h", "i", "hermitian"], "minShots": 0,
     "maxShots": 0},
    {"name": "Probability", "minShots": 0, "maxShots": 0},
    {"name": "Amplitude", "minShots": 0, "maxShots": 0},
    {"name": "AdjointGradient", "observables": ["x", "y", "z", "h", "i", "hermitian"],
     "minShots": 0, "maxShots": 0},
]
